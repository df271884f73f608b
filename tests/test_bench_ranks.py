"""The multi-rank plumbing of bench.py on CPU: world size 2 over gloo (127.0.0.1). Each rank reports
its own time; the job's number must come from the slowest rank, and the reference arm must print one
line from rank 0 only while the other ranks leave without work."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = 10.0 + 5.0 * rank  # rank r took 10 + 5 r ms
        t = bench.max_over_ranks(mine, "cpu")
        out.put((rank, t, bench.whole_job_qps(world, 4, 256, t)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, v in res:
        assert t == 15.0  # the slowest rank's time on every rank
        assert abs(v - 2 * 4 * 256 / 0.015) < 1e-6


def test_reference_arm_prints_once_under_torchrun():
    port = _free_port()
    env = dict(os.environ, OMP_NUM_THREADS="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--docs", "3000",
           "--queries", "16", "--cpu-queries", "4"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["e2e"]["h2d_bytes_per_step"] == 0 and rec["cpu_baseline"]["cores"] >= 1


def test_serving_sweep_record_with_and_without_graphs(monkeypatch):
    # the bench's serving bookkeeping on CPU, with a stand-in for the serving loop: warm-up at every
    # rate, one record per rate, capture counts split into warm-up and sweep only with graphs
    sys.path.insert(0, ROOT)
    import numpy as np

    import bench
    import hybridsearchsystem_b200 as hss

    calls = []

    class FakeServer:
        def __init__(self, table, **kw):
            self.graphs = kw.get("graphs")
            self.captures = 0

        def stats(self):
            return {"slots": 3, "completed": 0, "batches": 0, "mean_batch": 2.0, "p50_ms": 1.0, "p99_ms": 2.0,
                    "max_ms": 3.0, "graph_captures": self.captures, "graph_replays": 4 * self.captures,
                    "graph_capture_ms": 0.5 * self.captures}

        def set_threshold_model(self, model, margin):
            pass

        def reset_stats(self):
            pass

        def run_poisson(self, q, exprs, topks, rate, seed=0):
            calls.append((self.graphs, rate, len(q)))
            if self.graphs:
                self.captures += 2
            return np.ones(len(q)), rate, len(q) / rate

        def close(self):
            pass

    monkeypatch.setattr(hss, "Server", FakeServer)
    args = bench.parse_args([])
    ctx = {"table": None, "queries": np.zeros((64, 128), np.float32), "exprs": [""] * 64}
    rates = [1000.0, 50000.0, 200000.0]
    direct = bench.measure_serving(args, ctx, "bf16", rates, graphs=False)
    assert direct["graphs"] is None and [r["offered_qps"] for r in direct["rates"]] == [1000, 50000, 200000]
    graphs = bench.measure_serving(args, ctx, "bf16", rates, graphs=True)
    assert graphs["graphs"]["captures_in_warmup"] == 6 and graphs["graphs"]["captures_in_sweep"] == 6
    # a warm-up run at every rate before the timed ones, for each sweep
    assert [c[1] for c in calls[:3]] == rates and [c[1] for c in calls[3:6]] == rates
