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

Besides the headline form, one run measures (keys of the JSON line):
  forms              the chosen form with the learned threshold, the plain FP32 forms (TF32 tensor
                     cores, SIMT FFMA), the E4M3 form, batches of 64, and per-query K drawn from
                     {10, 100, 1000};
  parity_full_scale  every form's results for 256 queries at K = 10, 100 and 1000 against the
                     reference's own CpuTopKBatch (id sets, bit-exact FP32 scores, order);
  configs.cfg1       the one-segment configuration (131,072 docs, 64 tags, batches of 32) with its
                     parity against the reference;
  configs.cfg3       the precision form at 20M x 768 (FP32 + BF16 + E4M3 copies resident), recall and
                     score error against an FP64 dot product;
  serving            p50/p99 latency of the serving loop at open-loop Poisson rates.

--impl reference times the reference's own CPU ground-truth scan (CpuTopKBatch, compiled from the
reference sources into oracle/_ref) on this host's cores, on the same batch of queries per step.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
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
PARITY_KS = (10, 100, 1000)


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--docs", type=int, default=10_000_000)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--topk", type=int, default=100)
    ap.add_argument("--queries", type=int, default=2048, help="query pool the steps cycle through")
    ap.add_argument("--cpu-queries", type=int, default=0,
                    help="queries per reference step (0: one batch, fewer only if the run would exceed ~4 min)")
    ap.add_argument("--parity-queries", type=int, default=256, help="full-scale parity sample per K")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cand-cap", type=int, default=1 << 18, help="per-query candidate capacity")
    ap.add_argument("--sample-docs", type=int, default=32768, help="docs of the threshold sample per batch")
    ap.add_argument("--method", default="bf16", choices=list(METHODS),
                    help="the chosen form's candidate pass: simt (FP32 FFMA), tf32 (tensor cores over the FP32 "
                         "rows), bf16, e4m3")
    ap.add_argument("--learned", action="store_true", help="the chosen form uses the learned threshold")
    ap.add_argument("--train-queries", type=int, default=200_000, help="training queries of the learned threshold")
    ap.add_argument("--val-queries", type=int, default=10_000,
                    help="held-out queries of the learned threshold (early stop and margin)")
    ap.add_argument("--train-steps", type=int, default=4000, help="Adam steps (batches of 512) of the model")
    ap.add_argument("--margin-quantile", type=float, default=1.0,
                    help="quantile of the held-out (prediction - label) residuals taken as the margin")
    ap.add_argument("--no-learned-form", dest="learned_form", action="store_false",
                    help="skip measuring the chosen format with the learned threshold beside it")
    ap.add_argument("--no-plain", dest="plain", action="store_false",
                    help="skip measuring the plain FP32 (TF32) form beside the chosen one")
    ap.add_argument("--no-e4m3", dest="e4m3", action="store_false", help="skip measuring the E4M3 form")
    ap.add_argument("--no-serve", dest="serve", action="store_false", help="skip the serving-loop latency sweep")
    ap.add_argument("--no-batch64", dest="batch64", action="store_false",
                    help="skip measuring the chosen (and plain) form at batches of 64 queries")
    ap.add_argument("--no-kmix", dest="kmix", action="store_false",
                    help="skip measuring batches whose per-query K is drawn from {10, 100, 1000}")
    ap.add_argument("--no-cfg1", dest="cfg1", action="store_false", help="skip the one-segment configuration")
    ap.add_argument("--no-precision", dest="precision", action="store_false",
                    help="skip the 20M x 768 precision-form configuration")
    ap.add_argument("--precision-docs", type=int, default=20_000_000)
    ap.add_argument("--serve-requests", type=int, default=40000)
    ap.add_argument("--serve-rates", default="1000,10000,50000,100000,150000,200000",
                    help="offered Poisson rates (QPS) of the serving sweep")
    ap.add_argument("--serve-wait-us", type=int, default=300)
    ap.add_argument("--serve-slots", type=int, default=3, help="serving-loop slots (concurrent batches)")
    ap.add_argument("--no-graphs", dest="graphs", action="store_false",
                    help="end-to-end leg: launch every batch directly instead of replaying its captured CUDA "
                         "graph; serving: skip the sweep with graphs")
    ap.add_argument("--searchers", type=int, default=4,
                    help="searchers per form taking batches in turn, each on its own stream (at least 2)")
    return ap.parse_args(argv)


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


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


class ClockSampler:
    """SM clocks and clock-event reasons sampled in-process through NVML every 0.5 ms while running
    (the timed regions last tens of ms); nvidia-smi every 50 ms when NVML is unavailable. Only
    reads the GPU's state."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_uuid):
        self.uuid = gpu_uuid
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.source = None
        self._stop = threading.Event()
        self._thread = None
        self._proc = None
        self._out = None

    def _nvml_loop(self, nv, h):
        names = {nv.nvmlClocksEventReasonHwSlowdown: "hw_slowdown",
                 nv.nvmlClocksEventReasonHwThermalSlowdown: "hw_thermal_slowdown",
                 nv.nvmlClocksEventReasonSwThermalSlowdown: "sw_thermal_slowdown",
                 nv.nvmlClocksEventReasonSwPowerCap: "sw_power_cap"}
        while not self._stop.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                for bit, n in names.items():
                    if r & bit:
                        self.reasons.add(n)
            except Exception:
                break
            time.sleep(0.0005)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByUUID(self.uuid)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self._thread.start()
            self.source = "nvml 0.5 ms"
            while not self.samples and self._thread.is_alive():
                time.sleep(0.0005)
            self.samples.clear()  # the first sample predates the timed region
            self.reasons.clear()
            return self
        except Exception:
            self._thread = None
        self._out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self._proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                           "-lms", "50", "-i", self.uuid], stdout=self._out,
                                          stderr=subprocess.DEVNULL)
            self.source = "nvidia-smi 50 ms"
        except OSError:
            self._proc = None
        t0 = time.time()
        while self._proc and time.time() - t0 < 10 and os.path.getsize(self._out.name) == 0:
            time.sleep(0.01)
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=2)
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()

    def summary(self):
        if self._out is not None:
            self._out.flush()
            self._out.seek(0)
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for line in self._out.read().splitlines()[1:]:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    self.samples.append(float(parts[1]))
                    self.max_mhz = max(self.max_mhz or 0.0, float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        self.reasons.add(n)
            os.unlink(self._out.name)
            self._out = None
        return {"sm_mhz": float(np.median(self.samples)) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples), "source": self.source}


def reference_topk(vec, bits, queries, exprs, topk, threads=None):
    """The reference's CpuTopKBatch (oracle/_ref, compiled from its sources) on all host threads, or the
    oracle's restatement of it when the reference build is absent. Returns (ids [nq][topk] as sets in
    id order, counts, seconds, kind)."""
    import ctypes

    import oracle
    threads = threads or os.cpu_count() or 1
    nq = len(queries)
    q = np.ascontiguousarray(queries, np.float32)
    topks = np.full(nq, topk, np.int32)
    t0 = time.perf_counter()
    if oracle.ref_available():
        r = oracle.ref()
        arr = (ctypes.c_char_p * nq)(*[e.encode() for e in exprs])
        ids = np.full((nq, topk), -1, np.int64)
        counts = np.zeros(nq, np.int32)
        rc = r.ref_cpu_topk_batch(q.ctypes.data, nq, q.shape[1], arr, topks.ctypes.data, vec.ctypes.data,
                                  bits.ctypes.data, bits.shape[1] * 64, vec.shape[0], 0, 1, threads, topk,
                                  ids.ctypes.data, counts.ctypes.data)
        assert rc == 0
        kind = "reference"
    else:
        _, ids, counts = oracle.topk(q, list(exprs), topks, vec, bits, threads=threads, out_stride=topk)
        kind = "port"
    return ids, counts, time.perf_counter() - t0, kind


def cpu_record(nq, dt, kind, threads, topk, docs, batch_note=""):
    return {"value": nq / dt, "unit": "QPS", "cores": threads, "kind": kind, "cpu_model": cpu_model(),
            "sample": f"{nq} queries{batch_note} (filtered top-{topk}) over the full {docs}-doc corpus, "
                      f"CpuTopKBatch in {threads} query slices, fp32 mode"}


def ordered_truth(vec, queries, ids, counts):
    """The ground truth's ordered results from its id sets: each id's FP32 score in the ground truth's
    own arithmetic (sum over d ascending, every product and sum rounded to FP32, no contraction),
    sorted by (score desc, id asc). Returns a list of (scores, ids) per query."""
    out = []
    for i in range(len(counts)):
        c = int(counts[i])
        idv = np.sort(ids[i][:c].astype(np.int64))
        acc = np.zeros(c, np.float32)
        qv, dv = queries[i].astype(np.float32), vec[idv].astype(np.float32)
        for d in range(qv.shape[0]):
            acc = (acc + (qv[d] * dv[:, d]).astype(np.float32)).astype(np.float32)
        order = np.lexsort((idv, -acc.astype(np.float64)))
        out.append((acc[order], idv[order]))
    return out


def check_against(truth, scores, ids, counts):
    """Compares a form's results with the ordered ground truth: (id sets equal, scores bit-exact,
    order identical, queries that differ)."""
    sets = bits = order = True
    bad = 0
    for i, (ts, ti) in enumerate(truth):
        c = len(ti)
        if int(counts[i]) != c or set(ids[i][:c].tolist()) != set(ti.tolist()):
            sets = False
            bad += 1
            continue
        if not (ids[i][:c] == ti).all():
            order = False
            bad += 1
            continue
        if not (scores[i][:c].view(np.uint32) == ts.view(np.uint32)).all():
            bits = False
            bad += 1
    return sets, bits, order, bad


def run_reference(args):
    rank, local, world = dist_env()
    if rank != 0:
        return
    import torch
    device = "cuda" if torch.cuda.is_available() else None
    _, vec, bits, queries, exprs = workload(args, device)
    threads = os.cpu_count() or 1
    nq_pool = len(queries)
    # one batch of queries per step, as the GPU arm; fewer only when the run would take over ~4 min
    per_step = min(args.cpu_queries or args.batch, nq_pool)
    warm_n = max(1, min(per_step, 2 * threads))
    _, _, dt, _ = reference_topk(vec, bits, queries[:warm_n], exprs[:warm_n], args.topk, threads)
    rate = warm_n / dt
    if not args.cpu_queries and args.steps * per_step / rate > 240.0:
        per_step = max(threads, int(240.0 * rate / max(1, args.steps)))
    for w in range(max(0, args.warmup - 1)):
        reference_topk(vec, bits, queries[:warm_n], exprs[:warm_n], args.topk, threads)
    total_q, total_t, kind = 0, 0.0, "reference"
    for s in range(args.steps):
        a = (s * per_step) % max(1, nq_pool - per_step + 1)
        _, _, dt, kind = reference_topk(vec, bits, queries[a:a + per_step], exprs[a:a + per_step], args.topk,
                                        threads)
        total_t += dt
        total_q += per_step
    v = total_q / total_t
    note = f" per step (one batch of {args.batch})" if per_step == args.batch else \
        f" per step (batch {args.batch} cut to fit the run's time)"
    rec = cpu_record(per_step, total_t / args.steps, kind, threads, args.topk, args.docs, note)
    rec["value"] = v
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "QPS", "n_gpus": world,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_t / args.steps,
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                      "data": "synthetic (seeded cluster mixture, HYDSET2 shapes)",
                      "config": config_of(args, world), "cpu_baseline": rec,
                      "e2e": {"value": v, "unit": "QPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def form_name(method, learned):
    return FORMS[method] + (" + learned threshold" if learned else "")


def config_of(args, world):
    return {"workload": f"filtered top-{args.topk}, {args.docs} docs x 128 FP32, 256 tags, batch {args.batch}",
            "docs": args.docs, "dim": 128, "tags": 256, "batch": args.batch, "topk": args.topk,
            "doc_num_per_segment": 131072, "filters": "1-6 tags AND/OR/NOT, est. selectivity 1e-4..1",
            "parallelism": f"replica x{world}",
            "l2": "inputs larger than L2: every step reads the whole corpus copy (FP32 5.1 GB, BF16 2.6 GB, "
                  "E4M3 1.3 GB)",
            "form": form_name(args.method, args.learned), "method": args.method, "learned": args.learned}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def _topks(args, B, nb, kmode):
    """Per-batch K arrays: the headline K (kmode None), K drawn from {10, 100, 1000} per query
    ("mix"), or one K for every query (an int)."""
    if kmode is None:
        return [np.full(B, args.topk, np.uint32) for _ in range(nb)]
    if kmode != "mix":
        return [np.full(B, int(kmode), np.uint32) for _ in range(nb)]
    rng = np.random.default_rng(99)
    return [rng.choice(np.array(PARITY_KS, np.uint32), B) for _ in range(nb)]


def _kmode_note(kmode):
    if kmode is None:
        return ""
    return ", K from {10, 100, 1000} per query" if kmode == "mix" else f", K = {int(kmode)} for every query"


def trained_model(args, ctx, searcher, method):
    """The learned threshold model of a form's method, trained once per run on its own queries (seeded
    apart from the measured ones, the same selectivity range, K drawn from {10, 100, 1000}), labels
    from the exact path, with args.val_queries of them held out."""
    from hybridsearchsystem_b200.threshold import fit_threshold_model
    models = ctx.setdefault("models", {})
    if method not in models:
        n = args.train_queries + args.val_queries
        tq = ctx["mix"].queries(n, seed=20)
        te = data_filters(ctx["mix"], n, 21, pool_factor=4)  # a smaller pool keeps 210k draws to seconds
        tk = np.random.default_rng(22).choice([10, 100, 1000], n).astype(np.uint32)
        t0 = time.perf_counter()
        models[method] = fit_threshold_model(searcher, tq, te, tk, hidden=256, steps=args.train_steps, seed=3,
                                             n_val=args.val_queries, quantile=args.margin_quantile)
        models[method][2]["train_seconds"] = round(time.perf_counter() - t0, 1)
    return models[method]


def measure_form(args, ctx, method, learned=False, kmode=None, docs=None, dim=128, flush_l2=False,
                 e2e_direct=False):
    """One form of the path (candidate-pass method, with or without the learned threshold) over the
    context's workload: device-resident QPS (CUDA events, max over ranks), end-to-end QPS through the
    C-ABI, stage times and the candidate stage's roofline. With flush_l2 (a corpus that fits in L2),
    every step is timed on its own, after a 256 MB write that evicts L2 outside its events. Returns
    the record with the live searcher under "searcher" (for parity checks; the caller closes it)."""
    import torch

    import hybridsearchsystem_b200 as hss
    rank, world, dev, table = ctx["rank"], ctx["world"], ctx["dev"], ctx["table"]
    queries, exprs, barrier = ctx["queries"], ctx["exprs"], ctx["barrier"]
    docs = docs or args.docs
    B = args.batch
    kmax = args.topk if kmode is None else max(PARITY_KS)
    searcher = hss.FullRecallSearcher(table, max_batch=B, candidate_cap=args.cand_cap, method=METHODS[method],
                                      sample_docs=args.sample_docs)
    report = None
    if learned:
        model, margin, report = trained_model(args, ctx, searcher, method)
        searcher.set_threshold_model(model, margin)
    # args.searchers searchers of the same form: batch i runs on searcher i % D, so while the host
    # finishes one batch (its statuses, rare re-runs) the next ones are already queued.
    D = max(2, args.searchers)
    others = [hss.FullRecallSearcher(table, max_batch=B, candidate_cap=args.cand_cap, method=METHODS[method],
                                     sample_docs=args.sample_docs) for _ in range(D - 1)]
    if learned:
        for o in others:
            o.set_threshold_model(model, margin)
    searchers = (searcher, *others)
    for srch in searchers:
        srch.set_timing(True)
    nb = max(1, len(queries) // B)
    filters = [searcher.compile_filters(exprs[i * B:(i + 1) * B]) for i in range(nb)]
    topks = _topks(args, B, nb, kmode)
    d_q = torch.tensor(np.ascontiguousarray(queries[:nb * B]).reshape(nb, B, -1), device=dev)
    o_sc = torch.zeros((D, B, kmax), dtype=torch.float32, device=dev)
    o_id = torch.zeros((D, B, kmax), dtype=torch.int64, device=dev)
    o_n = torch.zeros((D, B), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream

    # Two ways to drive the two searchers: on one stream (a batch's stages run alone, so their event
    # times are the stage times and the candidate stage's roofline), or each on its own stream, so
    # that one batch's latency-bound stages (filter, sample threshold, select) overlap the other's
    # candidate pass: the throughput a caller gets from two searchers (the headline value).
    own_streams = [torch.cuda.Stream(device=dev) for _ in range(D)]
    mode = {"split": False}

    def stream_of(p):
        return own_streams[p] if mode["split"] else stream

    def enqueue(i, d_queries=None):
        j = (rank * 7919 + i) % nb
        p = i % D
        searchers[p].search_device_async(d_q[j].data_ptr() if d_queries is None else d_queries, B, filters[j],
                                         topks[j], o_sc[p].data_ptr(), o_id[p].data_ptr(), o_n[p].data_ptr(), kmax,
                                         stream_of(p).cuda_stream)

    def finish(i):
        srch = searchers[i % D]
        rc = srch.finish()
        assert rc == 0, srch.last_status(B)
        return srch.last_times()

    for i in range(args.warmup):
        enqueue(i)
        if i >= D - 1:
            finish(i - (D - 1))
    for i in range(max(0, args.warmup - (D - 1)), args.warmup):
        finish(i)
    torch.cuda.synchronize()
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev) if flush_l2 else None
    pairs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
             for _ in range(args.steps)] if flush_l2 else None
    # device-resident legs
    gpu_uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)

    def device_leg(split):
        """Times args.steps batches (events on the launching stream; with split, the default stream
        waits for both searchers' streams before the end event). Returns (ms, per-batch stage times,
        candidate stage times, launches, clocks)."""
        mode["split"] = split
        cand_ms, launches, stage_ms = [], 0, []
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(gpu_uuid) as clk:
            barrier()
            torch.cuda.synchronize()
            ev0.record(stream)
            for t2 in own_streams:
                t2.wait_stream(stream)

            def done(t):
                nonlocal launches
                cand_ms.append(t["candidates_ms"])
                stage_ms.append([t["filter_ms"], t["sample_ms"], t["candidates_ms"], t["select_ms"], t["total_ms"]])
                launches += t["launches"]

            for i in range(args.steps):
                if flush_l2:  # timed one step at a time, L2 written over between steps (no overlap)
                    flush.fill_(float(i))
                    pairs[i][0].record(stream)
                    enqueue(args.warmup + i)
                    done(finish(args.warmup + i))
                    pairs[i][1].record(stream)
                    continue
                enqueue(args.warmup + i)
                if i >= D - 1:
                    done(finish(args.warmup + i - (D - 1)))
            if not flush_l2:
                for i in range(max(0, args.steps - (D - 1)), args.steps):
                    done(finish(args.warmup + i))
            for t2 in own_streams:
                stream.wait_stream(t2)
            ev1.record(stream)
            torch.cuda.synchronize()
            barrier()
        own = sum(a.elapsed_time(b) for a, b in pairs) if flush_l2 else ev0.elapsed_time(ev1)
        mode["split"] = False
        return own, stage_ms, cand_ms, launches, clk.summary()

    # stage times and the roofline from the one-stream leg; the value from the two-stream leg (the
    # one-stream leg's when each step is timed alone)
    _, stage_ms, cand_ms, _, _ = device_leg(False)
    own_ms, _, _, launches, clocks = device_leg(False) if flush_l2 else device_leg(True)
    t_max = max_over_ranks(own_ms, dev)
    value = whole_job_qps(world, args.steps, B, t_max)

    # end-to-end leg through the C-ABI: pinned host queries in, results out, every step. Each step
    # is one batch through hss_filters_compile + hss_searcher_search_device_async / hss_searcher_finish
    # with its host->device query copy and device->host result copy, the two searchers alternating,
    # each on its own stream (one shared stream when each step is timed alone). A second host thread
    # compiles the next batch's filters (host-only work, table read-only) while this batch is on the
    # GPU; the ctypes calls release the interpreter lock.
    from concurrent.futures import ThreadPoolExecutor
    h_q = torch.tensor(np.ascontiguousarray(queries[:nb * B]).reshape(nb, B, -1)).pin_memory()
    h_sc = torch.zeros((D, B, kmax), dtype=torch.float32).pin_memory()
    h_id = torch.zeros((D, B, kmax), dtype=torch.int64).pin_memory()
    h_n = torch.zeros((D, B), dtype=torch.int32).pin_memory()
    d_stage = torch.zeros((D, B, dim), dtype=torch.float32, device=dev)
    out_ev = [torch.cuda.Event() for _ in range(D)]

    def batch_of(i):
        return (rank * 7919 + args.warmup + i) % nb

    # results go out on a copy stream that waits only for their own batch: on the compute stream they
    # would queue behind the next batch's kernels, and the host, waiting for them before it enqueues
    # the batch after, would leave the GPU idle between batches
    copy_stream = stream if flush_l2 else torch.cuda.Stream(device=dev)  # one step at a time: no overlap to gain
    done_ev = [torch.cuda.Event() for _ in range(D)]

    def e2e_run(steps, pool, ev=None):
        # per step: the next batch's filters compiled on a second host thread, its queries copied in
        # from pinned memory, the batch enqueued; then the previous batch finished and its results
        # copied out to pinned memory (read once its copy event has passed)
        fut = pool.submit(lambda: searcher.compile_filters(exprs[batch_of(0) * B:(batch_of(0) + 1) * B]))
        pending = []

        def retire(i, f):
            p = i % D
            rc = searchers[p].finish()
            assert rc == 0
            if copy_stream is stream:  # one step at a time: the copies follow the batch on its stream
                h_sc[p].copy_(o_sc[p], non_blocking=True)
                h_id[p].copy_(o_id[p], non_blocking=True)
                h_n[p].copy_(o_n[p], non_blocking=True)
                out_ev[p].record(stream)
                f.close()
                return
            if searchers[p].last_times()["retries"]:
                done_ev[p].record(ss[p])  # the re-runs ran behind later work on that stream
            copy_stream.wait_event(done_ev[p])
            with torch.cuda.stream(copy_stream):
                h_sc[p].copy_(o_sc[p], non_blocking=True)
                h_id[p].copy_(o_id[p], non_blocking=True)
                h_n[p].copy_(o_n[p], non_blocking=True)
                out_ev[p].record(copy_stream)
            f.close()

        for i in range(steps):
            j = batch_of(i)
            p = i % D
            f = fut.result()
            if i + 1 < steps:
                jn = batch_of(i + 1)
                fut = pool.submit(lambda jn=jn: searcher.compile_filters(exprs[jn * B:(jn + 1) * B]))
            if ev is not None:
                flush.fill_(float(i))
                ev[i][0].record(stream)
            out_ev[p].synchronize()  # this slot's previous results have reached the host
            if ss[p] is stream:
                d_stage[p].copy_(h_q[j], non_blocking=True)
            else:
                with torch.cuda.stream(ss[p]):
                    d_stage[p].copy_(h_q[j], non_blocking=True)
            searchers[p].search_device_async(d_stage[p].data_ptr(), B, f, topks[j], o_sc[p].data_ptr(),
                                             o_id[p].data_ptr(), o_n[p].data_ptr(), kmax, ss[p].cuda_stream)
            done_ev[p].record(ss[p])  # the batch's work as enqueued (re-runs, if any, come later)
            if ev is not None:  # one step at a time
                retire(i, f)
                stream.wait_event(out_ev[p])
                ev[i][1].record(stream)
                stream.synchronize()
                continue
            pending.append((i, f))
            if len(pending) == D:
                retire(*pending.pop(0))
        while pending:
            retire(*pending.pop(0))
        for e in out_ev:  # the timed region ends with the last results on the host
            stream.wait_event(e)
        stream.synchronize()

    # each searcher on its own stream, or (each step timed alone) all on the default stream
    ss = [stream] * D if flush_l2 else own_streams

    def timed_e2e(graphs):
        # graphs: each searcher replays its batch shape's captured CUDA graph (the default stream,
        # which one step at a time uses, cannot be captured); no stage timing in this leg
        for srch in searchers:
            srch.set_timing(False)
            srch.set_graphs(graphs)
        with ThreadPoolExecutor(1) as pool:
            e2e_run(2, pool)  # warm-up of the compile thread (and the graphs' captures)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            barrier()
            torch.cuda.synchronize()
            e0.record(stream)
            for t2 in own_streams:
                t2.wait_stream(stream)
            e2e_run(args.steps, pool, pairs)
            e1.record(stream)
            torch.cuda.synchronize()
            barrier()
        st = [srch.graph_stats() for srch in searchers]
        for srch in searchers:
            srch.set_graphs(False)
        assert not any(g["failed"] for g in st), st
        own = sum(a.elapsed_time(b) for a, b in pairs) if flush_l2 else e0.elapsed_time(e1)
        return (whole_job_qps(world, args.steps, B, max_over_ranks(own, dev)),
                {"captures": sum(g["captures"] for g in st), "replays": sum(g["replays"] for g in st)})

    use_graphs = args.graphs and not flush_l2
    e2e, graph_counts = timed_e2e(use_graphs)
    e2e_plain = timed_e2e(False)[0] if (e2e_direct and use_graphs) else None

    # roofline of the dominant stage, the candidate passes: algorithmic bytes per batch = the corpus
    # rows the passes read (docs x dim x element bytes, +4 B scale for E4M3; a learned form's
    # estimation pass re-reads a quarter) + the batch's filter bitmaps (B x docs/8 B)
    info = table.info
    words = info["segment_num"] * info["doc_num_per_segment"] // 64
    elem = {"simt": 4, "tf32": 4, "bf16": 2, "e4m3": 1}[method]
    reads = 1.25 if learned else 1.0
    alg_bytes = reads * docs * (dim * elem + (4 if method == "e4m3" else 0)) + B * words * 8
    cand_avg = float(np.mean(cand_ms))
    peaks = _peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg_bytes / (cand_avg / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "cand_traffic.json")
    if os.path.exists(tpath) and dim == 128:
        with open(tpath) as f:
            traffic = json.load(f).get(method)
    kernel = "cand_simt_kernel" if method == "simt" else ("tc2_cand_kernel" if B > 128 else "tc_cand_kernel")
    # the tensor side of the same stage: 2 d flops per (query, doc) pair of every pass, against the
    # pipe's peak (measured BF16 GEMM rate; TF32 and E4M3 by the nominal dense ratios 1/2 and 2)
    flops = reads * 2.0 * dim * docs * B
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
    out = {"value": value, "t_max_ms": t_max, "e2e": e2e, "batch": B, "roofline": roof, "clocks": clocks,
           "launches": launches, "e2e_graphs": graph_counts if use_graphs else None,
           "stages_ms": dict(zip(["filter", "sample", "candidates", "select", "total"],
                                 [round(float(x), 4) for x in np.mean(np.array(stage_ms), axis=0)])),
           "form": form_name(method, learned) + _kmode_note(kmode),
           "l2": "flushed between steps (256 MB write outside the step's events)" if flush_l2 else
                 "inputs larger than L2",
           "method": method, "learned": learned, "searcher": searcher, "dev": dev,
           "pipelined": f"{D} searchers of the form take batches in turn (enqueue batch i, then finish batch "
                        f"i - {D - 1}), each on its own stream so that one batch's filter, sample and select "
                        "overlap another's candidate pass (value, e2e); stages_ms and the roofline come from a "
                        "run of the same batches with the searchers on one stream, where stages do not "
                        "overlap"}
    if e2e_plain is not None:
        out["e2e_direct"] = e2e_plain  # the same leg with every batch launched directly
    for o in others:
        o.close()
    for f in filters:
        f.close()
    if report:
        out["model"], out["margin"] = model, margin
        out["learned_report"] = {k: (round(v, 5) if isinstance(v, float) else v) for k, v in report.items()}
        # what the model does on this workload, over measured batches: the docs each query's candidate
        # passes kept (what the select step reads) without the model and with it, and the queries
        # whose predicted threshold was too high (re-run at a proven threshold)
        plain, with_model, miss, kk = [], [], [], []
        for j in range(min(nb, 16)):
            f = searcher.compile_filters(exprs[j * B:(j + 1) * B])
            for m in (None, model):
                searcher.set_threshold_model(m, margin)
                rc = searcher.search_device(d_q[j].data_ptr(), B, f, topks[j], o_sc.data_ptr(), o_id.data_ptr(),
                                            o_n.data_ptr(), kmax, sh)
                assert rc == 0
                (with_model if m else plain).append(searcher.last_candidate_counts(B).astype(np.int64))
            miss.append(searcher.last_threshold_misses(B))
            f.close()
            kk.append(topks[j].astype(np.int64))
        plain, with_model, miss, kk = (np.concatenate(plain), np.concatenate(with_model), np.stack(miss),
                                       np.concatenate(kk))
        searcher.set_threshold_model(model, margin)
        by_k = {}
        for k in sorted(set(kk.tolist())):
            sel = kk == k
            by_k[f"K{k}"] = {"candidates_without_model": int(plain[sel].sum()),
                             "candidates_with_model": int(with_model[sel].sum()),
                             "miss_rate": round(float(miss.reshape(-1)[sel].mean()), 5)}
        out["learned_report"].update({
            "candidates_without_model": int(plain.sum()), "candidates_with_model": int(with_model.sum()),
            "pruned_fraction": round(1.0 - with_model.sum() / max(1, plain.sum()), 4),
            "miss_rate": round(float(miss.mean()), 5),
            "batches_with_a_miss": round(float(miss.any(axis=1).mean()), 4), "queries": int(len(kk)),
            "by_k": by_k})
    return out


def parity_of_form(searcher, dev, B, pq, pe, truth_by_k):
    """Runs a form's searcher over the parity queries at every K (batches of B) and checks each K's
    results against the reference's ordered ground truth."""
    import torch
    res = {}
    n = len(pq)
    for k, truth in truth_by_k.items():
        d_q = torch.tensor(np.ascontiguousarray(pq), device=dev)
        o_sc = torch.zeros((B, k), dtype=torch.float32, device=dev)
        o_id = torch.zeros((B, k), dtype=torch.int64, device=dev)
        o_n = torch.zeros(B, dtype=torch.int32, device=dev)
        sc_all = np.zeros((n, k), np.float32)
        id_all = np.zeros((n, k), np.int64)
        n_all = np.zeros(n, np.int64)
        sh = torch.cuda.current_stream().cuda_stream
        for a in range(0, n, B):
            b = min(n, a + B)
            f = searcher.compile_filters(pe[a:b])
            rc = searcher.search_device(d_q[a].data_ptr(), b - a, f, np.full(b - a, k, np.uint32), o_sc.data_ptr(),
                                        o_id.data_ptr(), o_n.data_ptr(), k, sh)
            torch.cuda.synchronize()
            f.close()
            assert rc == 0, searcher.last_status(b - a)
            sc_all[a:b] = o_sc.cpu().numpy()[:b - a]
            id_all[a:b] = o_id.cpu().numpy()[:b - a]
            n_all[a:b] = o_n.cpu().numpy()[:b - a]
        sets, bits, order, bad = check_against(truth, sc_all, id_all, n_all)
        res[f"K{k}"] = {"id_sets_match": sets, "scores_bit_exact": bits, "order_score_desc_id_asc": order,
                        "queries_differing": bad}
        res.setdefault("_last", (sc_all, id_all, n_all))
    last = res.pop("_last")
    return res, last


def fp64_error(vec, queries, scores, ids, counts):
    """Max and median |returned FP32 score - FP64 dot product of the same vectors|."""
    ea, er = [], []
    for i in range(len(counts)):
        c = int(counts[i])
        if c == 0:
            continue
        ex = vec[ids[i][:c]].astype(np.float64) @ queries[i].astype(np.float64)
        e = np.abs(scores[i][:c].astype(np.float64) - ex)
        ea.append(e)
        er.append(e / np.maximum(np.abs(ex), 1e-30))
    if not ea:
        return None
    ea, er = np.concatenate(ea), np.concatenate(er)
    return {"max_abs": float(ea.max()), "median_abs": float(np.median(ea)), "max_rel": float(er.max()),
            "median_rel": float(np.median(er))}


def data_filters(mix, n, seed, pool_factor=24):
    from hybridsearchsystem_b200 import data
    return data.make_filters(mix, n, n_tags=(1, 6), seed=seed, selectivity_range=(1e-4, 1.0),
                             pool_factor=pool_factor)


def measure_serving(args, ctx, method, rates, model=None, margin=0.0, graphs=True):
    """p50/p99 latency of single queries through the serving loop (continuous batching) at open-loop
    Poisson arrival rates. Requests mix the workload's filters (selectivity log-uniform in
    [1e-4, 1]) with per-request K log-uniform in [1, 1000]. graphs: the slots replay each batch
    shape's captured CUDA graph."""
    import hybridsearchsystem_b200 as hss
    srv = hss.Server(ctx["table"], slots=args.serve_slots, max_batch=args.batch, max_wait_us=args.serve_wait_us,
                     method=METHODS[method], candidate_cap=args.cand_cap, graphs=graphs)
    if model is not None:
        srv.set_threshold_model(model, margin)
    srv_slots = srv.stats()["slots"]  # admitted within the device-memory budget
    q, ex = ctx["queries"], ctx["exprs"]
    kk = np.exp(np.random.default_rng(77).uniform(0.0, np.log(1000.0), len(q))).astype(np.uint32) + 1
    kk = np.minimum(kk, 1000)
    # warm-up at every rate of the sweep (with graphs, the batch shapes each load level forms are
    # captured once, as in a server that runs for long), not timed
    for i, rate in enumerate(rates):
        n = int(min(20000, max(2000, rate * 0.1)))
        idx = (np.arange(n) + 7919 * (i + 1)) % len(q)
        srv.run_poisson(q[idx], [ex[i] for i in idx], kk[idx], rate, seed=i + 1)
    warm = srv.stats()
    out = []
    for rate in rates:
        n = int(min(args.serve_requests, max(2000, rate * 0.5)))
        idx = np.arange(n) % len(q)
        srv.reset_stats()
        lat, offered, wall = srv.run_poisson(q[idx], [ex[i] for i in idx], kk[idx], rate, seed=int(rate))
        st = srv.stats()
        out.append({"offered_qps": round(offered), "completed_qps": round(n / wall), "p50_ms": round(st["p50_ms"], 3),
                    "p99_ms": round(st["p99_ms"], 3), "mean_batch": round(st["mean_batch"], 1)})
    st = srv.stats()
    srv.close()
    graph = None
    if graphs:
        graph = {"captures_in_warmup": warm["graph_captures"],
                 "captures_in_sweep": st["graph_captures"] - warm["graph_captures"],
                 "replays_in_sweep": st["graph_replays"] - warm["graph_replays"],
                 "capture_ms_per_shape": round(st["graph_capture_ms"] / max(1, st["graph_captures"]), 3)}
    return {"form": form_name(method, model is not None), "slots": srv_slots, "graphs": graph,
            "max_wait_us": args.serve_wait_us, "topk": "log-uniform in [1, 1000] per request",
            "warmup": "at each rate, max(2000, 0.1 s of) requests (not timed)", "rates": out}


def summary(f, steps):
    d = {"value": f["value"], "e2e_qps": f["e2e"], "ms_per_step": f["t_max_ms"] / steps,
         "stages_ms": f["stages_ms"], "roofline_frac": f["roofline"]["frac"], "form": f["form"],
         "batch": f["batch"], "l2": f["l2"], "clocks": {k: f["clocks"][k] for k in ("sm_mhz", "reasons", "samples")}}
    if f.get("e2e_graphs"):
        d["e2e_graphs"] = f["e2e_graphs"]
    if "e2e_direct" in f:
        d["e2e_direct_qps"] = f["e2e_direct"]
    if "learned_report" in f:
        d["learned_report"] = f["learned_report"]
    if "parity" in f:
        d["parity"] = f["parity"]
    return d


def run_cfg1(args, dev, local):
    """The one-segment configuration: 131,072 docs x 128, 64 tags (densities in [1e-3, 0.5]), filters
    of 1-4 tags, 1,000 queries in batches of 32, top-100; chosen and plain forms, each checked against
    the reference on all 1,000 queries."""
    import copy

    import hybridsearchsystem_b200 as hss
    from hybridsearchsystem_b200 import data
    c = data.CONFIGS["cfg1"]
    mix = data.Mixture(c["dim"], c["tag_num"], c["p_range"], n_clusters=1024, sigma=0.3, n_corr=16, seed=5)
    vec, bits, _ = mix.corpus(c["n"], seed=51)
    queries = mix.queries(c["nq"], seed=52)
    exprs = data.make_filters(mix, c["nq"], n_tags=c["n_tags"], seed=53)
    table = hss.DataTable.build(vec, bits, c["tag_num"], device=local, doc_num_per_segment=c["doc_num_per_segment"])
    threads = os.cpu_count() or 1
    ids, counts, dt, kind = reference_topk(vec, bits, queries, exprs, 100, threads)
    truth = {100: ordered_truth(vec, queries, ids, counts)}
    a = copy.copy(args)
    a.batch, a.topk, a.docs = c["batch"], 100, c["n"]
    a.steps = max(args.steps, 31)
    ctx = {"rank": 0, "world": 1, "dev": dev, "table": table, "queries": queries, "exprs": exprs,
           "barrier": lambda: None}
    out = {"workload": "filtered top-100, 131072 docs x 128 FP32 (one segment), 64 tags, batch 32",
           "cpu_baseline": cpu_record(len(queries), dt, kind, threads, 100, c["n"])}
    for key, method in (("chosen", args.method), ("plain_fp32", "tf32"), ("plain_fp32_simt", "simt")):
        f = measure_form(a, ctx, method, flush_l2=True)
        f["parity"], _ = parity_of_form(f["searcher"], dev, a.batch, queries, exprs, truth)
        f["searcher"].close()
        out[key] = summary(f, a.steps)
    table.close()
    return out


def run_cfg3(args, dev, local):
    """The precision form at 20M x 768: FP32 rows (61 GB) with BF16 and E4M3 copies resident together
    (108 GB), 64 tags, batches of 256, top-100. Each form's QPS, recall against the reference's
    CpuTopKBatch (run over the corpus in 1M-doc chunks copied to the host, merged by (score desc, id
    asc)) for a query sample, and the returned scores' error against an FP64 dot product."""
    import copy

    import torch

    import hybridsearchsystem_b200 as hss
    from hybridsearchsystem_b200 import data
    n, dim, tags = args.precision_docs, 768, 64
    mix = data.Mixture(dim, tags, (1e-3, 0.5), n_clusters=1024, sigma=0.3, n_corr=16, seed=7)
    t0 = time.perf_counter()
    d_vec, bits = mix.corpus_device(n, device=dev, seed=71)
    table = hss.DataTable.build_device(d_vec.data_ptr(), n, dim, bits, tags, device=local,
                                       doc_num_per_segment=131072)
    queries = mix.queries(2048, seed=72)
    exprs = data.make_filters(mix, 2048, n_tags=(1, 4), seed=73)
    # reference ground truth for a sample, in chunks of the corpus copied to the host
    npar = 32
    threads = os.cpu_count() or 1
    chunk = 1 << 20
    best = [[] for _ in range(npar)]
    t_ref = 0.0
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        hv = d_vec[a:b].cpu().numpy()
        ids, counts, dt, kind = reference_topk(hv, bits[a:b], queries[:npar], exprs[:npar], 100, threads)
        t_ref += dt
        for i in range(npar):
            c = int(counts[i])
            loc = np.sort(ids[i][:c])
            acc = np.zeros(c, np.float32)
            for d in range(dim):
                acc = (acc + (queries[i][d] * hv[loc, d]).astype(np.float32)).astype(np.float32)
            best[i].extend(zip((-acc.astype(np.float64)).tolist(), (loc + a).tolist(), acc.tolist()))
        del hv
    truth = []
    for i in range(npar):
        top = sorted(best[i])[:100]
        truth.append((np.array([t[2] for t in top], np.float32), np.array([t[1] for t in top], np.int64)))
    # the truth's rows on the host, for the FP64 error of the returned scores
    want = np.unique(np.concatenate([t[1] for t in truth]))
    rows64 = d_vec[torch.tensor(want, device=dev)].cpu().numpy().astype(np.float64)
    del d_vec
    torch.cuda.empty_cache()
    build_s = time.perf_counter() - t0
    a = copy.copy(args)
    a.docs, a.topk, a.batch = n, 100, 256
    a.steps = min(args.steps, 10)
    ctx = {"rank": 0, "world": 1, "dev": dev, "table": table, "queries": queries, "exprs": exprs,
           "barrier": lambda: None}
    out = {"workload": f"filtered top-100, {n} docs x {dim} FP32 + BF16 + E4M3 copies, {tags} tags, batch 256",
           "setup_s": round(build_s, 1),
           "cpu_baseline": {"value": npar / t_ref, "unit": "QPS", "cores": threads, "kind": kind,
                            "cpu_model": cpu_model(),
                            "sample": f"{npar} queries over the corpus in 1M-doc chunks"}}
    pos = {int(g): j for j, g in enumerate(want)}
    for method in ("tf32", "bf16", "e4m3"):
        f = measure_form(a, ctx, method, docs=n, dim=dim)
        par, (sc, ids, cnt) = parity_of_form(f["searcher"], dev, a.batch, queries[:npar], exprs[:npar],
                                             {100: truth})
        f["parity"] = par
        f["searcher"].close()
        s = summary(f, a.steps)
        # recall of the reference's ids and the FP64 error of the returned scores
        rec = [len(set(ids[i][:len(truth[i][1])].tolist()) & set(truth[i][1].tolist())) / max(1, len(truth[i][1]))
               for i in range(npar)]
        s["recall"] = float(np.mean(rec))
        ea = []
        for i in range(npar):
            c = int(cnt[i])
            rows = np.array([pos.get(int(g), -1) for g in ids[i][:c]])
            if c == 0 or (rows < 0).any():
                continue
            ex = rows64[rows] @ queries[i].astype(np.float64)
            ea.append(np.abs(sc[i][:c].astype(np.float64) - ex))
        if ea:
            ea = np.concatenate(ea)
            s["score_error_vs_fp64"] = {"max_abs": float(ea.max()), "median_abs": float(np.median(ea))}
        out[method] = s
    table.close()
    return out


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
    solo = rank == 0 and world == 1
    # the reference's ground truth for the parity sample (K = 10, 100, 1000); the K = 100 run is the
    # timed CPU baseline
    truth, cb = None, None
    if solo and not args.no_cpu_baseline:
        npq = min(args.parity_queries, len(queries))
        pq, pe = queries[:npq], exprs[:npq]
        threads = os.cpu_count() or 1
        truth = {}
        for k in PARITY_KS:
            ids, counts, dt, kind = reference_topk(vec, bits, pq, pe, k, threads)
            truth[k] = ordered_truth(vec, pq, ids, counts)
            if k == K:
                cb = cpu_record(npq, dt, kind, threads, K, args.docs)

    forms = {}

    def run_form(key, method, learned=False, batch=None, kmode=None):
        import copy
        a = args
        if batch and batch != args.batch:
            a = copy.copy(args)
            a.batch = batch
        f = measure_form(a, ctx, method, learned=learned, kmode=kmode, e2e_direct=key == "chosen")
        if truth is not None and kmode is None:
            f["parity"], last = parity_of_form(f["searcher"], dev, a.batch, pq, pe, truth)
            if key == "chosen":
                f["fp64"] = fp64_error(vec, pq, *last)
        if key != "chosen":
            f["searcher"].close()
            f.pop("searcher")
        forms[key] = f
        return f

    chosen = run_form("chosen", args.method, learned=args.learned)
    if args.learned_form and not args.learned:
        run_form("chosen_learned", args.method, learned=True)
    if args.plain:
        # the two plain FP32 forms (both read the FP32 rows): TF32 tensor cores, and SIMT FFMA
        if not (args.method == "tf32" and not args.learned):
            run_form("plain_fp32", "tf32")
        run_form("plain_fp32_simt", "simt")
    if args.e4m3 and args.method != "e4m3":
        run_form("e4m3", "e4m3")
    if args.batch64 and args.batch != 64:
        # the configuration's other batch size: 64 queries per batch (one SM per 128-doc tile)
        run_form("chosen_batch64", args.method, batch=64)
        if args.plain:
            run_form("plain_fp32_batch64", "tf32", batch=64)
    if args.kmix:
        run_form("chosen_kmix", args.method, kmode="mix")
        if args.learned_form and not args.learned:
            run_form("chosen_learned_kmix", args.method, learned=True, kmode="mix")
        if args.plain:
            run_form("plain_fp32_kmix", "tf32", kmode="mix")
        # the K = 1000 slice, where the doc sample's threshold is loosest
        run_form("chosen_k1000", args.method, kmode=1000)
        if args.learned_form and not args.learned:
            run_form("chosen_learned_k1000", args.method, learned=True, kmode=1000)
    serving = None
    if solo and args.serve:
        rates = [float(r) for r in args.serve_rates.split(",")]
        # each form's sweep with every batch launched directly; the chosen form's also with the slots
        # replaying captured CUDA graphs (a capture now and then took tens of ms of host time, which
        # shows in that sweep's p99)
        serving = {"chosen": measure_serving(args, ctx, args.method, rates, chosen.get("model"),
                                             chosen.get("margin", 0.0), graphs=False)}
        if args.graphs:
            serving["chosen_graphs"] = measure_serving(args, ctx, args.method, rates, chosen.get("model"),
                                                       chosen.get("margin", 0.0), graphs=True)
        if "chosen_learned" in forms:
            serving["chosen_learned"] = measure_serving(args, ctx, args.method, rates, forms["chosen_learned"]["model"],
                                                        forms["chosen_learned"]["margin"], graphs=False)
        if args.plain:
            serving["plain_fp32"] = measure_serving(args, ctx, "tf32", rates, graphs=False)

    rec = {"metric": METRIC, "value": chosen["value"], "unit": "QPS", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": chosen["t_max_ms"] / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": {"simt": "f32", "tf32": "f32", "bf16": "bf16",
                                                             "e4m3": "e4m3"}[args.method] + "+f32 rescore",
           "data": "synthetic (seeded cluster mixture, HYDSET2 shapes)",
           "config": config_of(args, world),
           "e2e": {"value": chosen["e2e"], "unit": "QPS", "h2d_bytes_per_step": B * 128 * 4,
                   "d2h_bytes_per_step": B * K * (4 + 8) + B * 4,
                   "path": "hss_filters_compile (next batch, compile thread) + hss_searcher_search_device_async / "
                           f"hss_searcher_finish per batch ({max(2, args.searchers)} searchers taking batches in "
                           "turn, each on its own stream"
                           + (", each batch's first attempt replayed from its shape's captured CUDA graph"
                              if args.graphs else "") + "), pinned host queries in, results out on a copy stream"},
           "roofline": chosen["roofline"], "clocks": chosen["clocks"], "gpu_launches": chosen["launches"],
           "stages_ms": chosen["stages_ms"], "forms": {k: summary(v, args.steps) for k, v in forms.items()}}
    if "plain_fp32" in forms:
        rec["chosen_over_plain"] = chosen["value"] / forms["plain_fp32"]["value"]
    if serving:
        rec["serving"] = serving
    if cb is not None:
        rec["cpu_baseline"] = cb
        per = {k: v["parity"] for k, v in forms.items() if "parity" in v}
        ok = all(all(x["id_sets_match"] and x["scores_bit_exact"] and x["order_score_desc_id_asc"]
                     for x in p.values()) for p in per.values())
        rec["parity_full_scale"] = {"queries": len(pq), "k": list(PARITY_KS), "against": cb["kind"],
                                    "all_forms_exact": ok, "forms": per,
                                    "score_error_vs_fp64": chosen.get("fp64")}
    chosen["searcher"].close()
    for f in forms.values():
        for key in ("searcher", "model"):
            f.pop(key, None)
    configs = {}
    if solo and args.cfg1:
        configs["cfg1"] = run_cfg1(args, dev, local)
    if solo and args.precision:
        table.close()
        del vec, bits
        torch.cuda.empty_cache()
        configs["cfg3"] = run_cfg3(args, dev, local)
    if configs:
        rec["configs"] = configs
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
