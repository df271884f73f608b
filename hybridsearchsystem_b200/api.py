"""Python mirror of the reference's host API for the filtered full-recall path.

    DataTable            DataTable::LoadData / the offline builder (src/engine/index/data_table.h)
    FullRecallSearcher   AddQuery + BatchSearch (src/engine/retrieval/searcher/full_recall_searcher.h)
    operators            the device operators' launch entry points (include/hss.h)

Device pointers are passed as integers (``tensor.data_ptr()``); streams as integers
(``torch.cuda.current_stream().cuda_stream``) or 0 for the default stream. Everything runs through
libhss.so; nothing here computes results on the CPU.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check


def _np_ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class DataTable:
    """Index resident on one GPU (device < 0: host only, for building / compiling / saving)."""

    def __init__(self, handle, device):
        self._h = ctypes.c_void_p(handle)
        self.device = device

    @classmethod
    def build(cls, vectors, tag_bits, tag_num, device=0, doc_num_per_segment=131072, density_threshold=1.0 / 64,
              matrix_posting=False, sparse_packed=False, doc_offset=0):
        lib = _lib.load()
        vectors = np.ascontiguousarray(vectors, dtype=np.float32)
        tag_bits = np.ascontiguousarray(tag_bits, dtype=np.uint64)
        n, dim = vectors.shape
        assert tag_bits.shape[0] == n and tag_bits.shape[1] == (tag_num + 63) // 64
        cfg = _lib.IndexConfig(doc_num_per_segment, density_threshold, int(matrix_posting), int(sparse_packed),
                               doc_offset)
        h = ctypes.c_void_p()
        check(lib.hss_table_build(device, _np_ptr(vectors), _np_ptr(tag_bits), n, dim, tag_num, ctypes.byref(cfg),
                                  ctypes.byref(h)))
        return cls(h.value, device)

    @classmethod
    def build_device(cls, d_vectors, doc_num, dim, tag_bits, tag_num, device=0, doc_num_per_segment=131072,
                     density_threshold=1.0 / 64, matrix_posting=False, sparse_packed=False, doc_offset=0):
        """The same build from vectors already on `device` (d_vectors: device pointer of [doc_num][dim]
        float32, copied by the table; the caller may free it afterwards). tag_bits is a host array."""
        lib = _lib.load()
        tag_bits = np.ascontiguousarray(tag_bits, dtype=np.uint64)
        assert tag_bits.shape[0] == doc_num and tag_bits.shape[1] == (tag_num + 63) // 64
        cfg = _lib.IndexConfig(doc_num_per_segment, density_threshold, int(matrix_posting), int(sparse_packed),
                               doc_offset)
        h = ctypes.c_void_p()
        check(lib.hss_table_build_device(device, ctypes.c_void_p(d_vectors), _np_ptr(tag_bits), doc_num, dim, tag_num,
                                         ctypes.byref(cfg), ctypes.byref(h)))
        return cls(h.value, device)

    @classmethod
    def load(cls, directory, device=0):
        lib = _lib.load()
        h = ctypes.c_void_p()
        check(lib.hss_table_load(device, str(directory).encode(), ctypes.byref(h)))
        return cls(h.value, device)

    def save(self, directory):
        check(_lib.load().hss_table_save(self._h, str(directory).encode()))

    @classmethod
    def load_reference(cls, directory, device=0):
        """An index directory in the reference's own layout (its fr_builder's output)."""
        lib = _lib.load()
        h = ctypes.c_void_p()
        check(lib.hss_table_load_reference(device, str(directory).encode(), ctypes.byref(h)))
        return cls(h.value, device)

    def save_reference(self, directory, split_doc_num_zn=16):
        """Writes the table in the reference's index layout (FP16 vectors in Zn blocks)."""
        check(_lib.load().hss_table_save_reference(self._h, str(directory).encode(), split_doc_num_zn))

    @property
    def load_times(self):
        """Where the last load spent its time (ms) and the bytes it moved."""
        ms = np.zeros(6, np.float64)
        vb, pb = ctypes.c_uint64(), ctypes.c_uint64()
        th = ctypes.c_uint32()
        check(_lib.load().hss_table_load_times(self._h, _np_ptr(ms), ctypes.byref(vb), ctypes.byref(pb),
                                               ctypes.byref(th)))
        return {"meta_ms": ms[0], "postings_read_ms": ms[1], "vectors_read_ms": ms[2], "vectors_h2d_ms": ms[3],
                "postings_h2d_ms": ms[4], "total_ms": ms[5], "vector_bytes": vb.value, "posting_bytes": pb.value,
                "threads": th.value}

    def close(self):
        if self._h:
            _lib.load().hss_table_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def info(self):
        n = ctypes.c_uint64()
        dim, segs, p, rows = (ctypes.c_uint32() for _ in range(4))
        mx = ctypes.c_float()
        check(_lib.load().hss_table_info(self._h, ctypes.byref(n), ctypes.byref(dim), ctypes.byref(segs),
                                         ctypes.byref(p), ctypes.byref(rows), ctypes.byref(mx)))
        return {"doc_num": n.value, "dim": dim.value, "segment_num": segs.value, "doc_num_per_segment": p.value,
                "posting_rows": rows.value, "max_norm": mx.value}

    def posting(self, token, segment):
        """Host bytes of a token's posting in one segment, or None when the token is absent there."""
        data = _lib.c_u8p()
        n = ctypes.c_uint32()
        check(_lib.load().hss_table_posting(self._h, token, segment, ctypes.byref(data), ctypes.byref(n)))
        if not data or n.value == 0:
            return None
        return bytes(ctypes.string_at(data, n.value))

    def device_ptrs(self):
        v, t, g = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(_lib.load().hss_table_device_ptrs(self._h, ctypes.byref(v), ctypes.byref(t), ctypes.byref(g)))
        return v.value, t.value, g.value

    def compile_filter(self, expr):
        """(postfix program, operand rows, opNum, empty_tree) of one filter text."""
        prog = np.zeros(_lib.HSS_MAX_PROGRAM * 4, np.uint32)
        rows = np.zeros(_lib.HSS_MAX_OPERANDS * 4, np.uint32)
        pl, rl, opn = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        empty = ctypes.c_int32()
        check(_lib.load().hss_filter_compile(self._h, expr.encode(), _np_ptr(prog), prog.size, ctypes.byref(pl),
                                             _np_ptr(rows), rows.size, ctypes.byref(rl), ctypes.byref(opn),
                                             ctypes.byref(empty)))
        return prog[:pl.value].copy(), rows[:rl.value].copy(), opn.value, bool(empty.value)


class Filters:
    """A batch's filter texts compiled once (TextFilter::PrepareExpr)."""

    def __init__(self, searcher, exprs):
        lib = _lib.load()
        arr = (ctypes.c_char_p * max(1, len(exprs)))(*[e.encode() for e in exprs])
        h = ctypes.c_void_p()
        check(lib.hss_filters_compile(searcher._h, arr, len(exprs), ctypes.byref(h)))
        self._h = h
        self.n = len(exprs)

    def close(self):
        if self._h:
            _lib.load().hss_filters_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FullRecallSearcher:
    def __init__(self, table, max_batch=256, candidate_cap=1 << 18, sample_docs=32768, max_retries=4, method=0,
                 decode_in_place=False, workspace=None):
        """workspace: (device pointer, bytes) of a caller-owned arena of at least workspace_bytes(...)
        bytes (hss_searcher_create_in); None lets the searcher allocate its own."""
        lib = _lib.load()
        self.table = table
        self.dim = table.info["dim"]
        cfg = _lib.SearcherConfig(max_batch, candidate_cap, sample_docs, max_retries, method, int(decode_in_place))
        h = ctypes.c_void_p()
        if workspace is None:
            check(lib.hss_searcher_create(table._h, ctypes.byref(cfg), ctypes.byref(h)))
        else:
            check(lib.hss_searcher_create_in(table._h, ctypes.byref(cfg), ctypes.c_void_p(workspace[0]),
                                             workspace[1], ctypes.byref(h)))
        self._h = h
        self.max_batch = max_batch
        self._pending = 0

    @staticmethod
    def workspace_bytes(table, max_batch=256, candidate_cap=1 << 18, sample_docs=32768, max_retries=4, method=0,
                        decode_in_place=False):
        """Device bytes of one searcher's arena for this table and configuration."""
        cfg = _lib.SearcherConfig(max_batch, candidate_cap, sample_docs, max_retries, method, int(decode_in_place))
        return _lib.load().hss_searcher_workspace_bytes(table._h, ctypes.byref(cfg))

    @staticmethod
    def prepare_table(table, max_batch=256, candidate_cap=1 << 18, sample_docs=32768, max_retries=4, method=0,
                      decode_in_place=False):
        """Builds the table's resident data a searcher of this configuration reads (hss_table_prepare)."""
        cfg = _lib.SearcherConfig(max_batch, candidate_cap, sample_docs, max_retries, method, int(decode_in_place))
        check(_lib.load().hss_table_prepare(table._h, ctypes.byref(cfg)))

    def close(self):
        if self._h:
            _lib.load().hss_searcher_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_query(self, filter_expr, vector, topk):
        v = np.ascontiguousarray(vector, dtype=np.float32)
        check(_lib.load().hss_searcher_add_query(self._h, (filter_expr or "").encode(), _np_ptr(v), v.size, topk))
        self._pending += 1

    def batch_search(self, out_stride=None):
        """Runs the added queries. Returns (scores [n][stride], ids [n][stride], counts [n])."""
        n = self._pending
        stride = out_stride or _lib.HSS_MAX_TOPK
        scores = np.zeros((max(n, 1), stride), np.float32)
        ids = np.full((max(n, 1), stride), -1, np.int64)
        counts = np.zeros(max(n, 1), np.uint32)
        self._pending = 0
        rc = _lib.load().hss_searcher_batch_search(self._h, _np_ptr(scores), _np_ptr(ids), _np_ptr(counts), stride)
        if rc != _lib.HSS_ERR_QUERY:
            check(rc)
        return scores[:n], ids[:n], counts[:n]

    def compile_filters(self, exprs):
        return Filters(self, exprs)

    def search_device(self, d_queries, nq, filters, topks, d_scores, d_ids, d_counts, out_stride, stream=0):
        """Device-resident batch. Returns the status code (HSS_OK or HSS_ERR_QUERY)."""
        t = np.ascontiguousarray(topks, dtype=np.uint32)
        rc = _lib.load().hss_searcher_search_device(self._h, d_queries, nq, filters._h, _np_ptr(t), d_scores, d_ids,
                                                    d_counts, out_stride, stream)
        if rc != _lib.HSS_ERR_QUERY:
            check(rc)
        return rc

    def search_device_async(self, d_queries, nq, filters, topks, d_scores, d_ids, d_counts, out_stride, stream=0):
        """Enqueues a device-resident batch and returns at once; finish() completes it."""
        t = np.ascontiguousarray(topks, dtype=np.uint32)
        check(_lib.load().hss_searcher_search_device_async(self._h, d_queries, nq, filters._h, _np_ptr(t), d_scores,
                                                           d_ids, d_counts, out_stride, stream))

    def finish(self):
        """Waits for the enqueued batch (re-running overflowed queries). Returns HSS_OK or HSS_ERR_QUERY."""
        rc = _lib.load().hss_searcher_finish(self._h)
        if rc != _lib.HSS_ERR_QUERY:
            check(rc)
        return rc

    def filter_device(self, filters, nq, d_bits, stride_words, d_pass=None, stream=0):
        """Filter stage alone: per-query doc bitmaps into d_bits. Returns the status code."""
        rc = _lib.load().hss_searcher_filter_device(self._h, filters._h, nq, d_bits, stride_words, d_pass, stream)
        if rc != _lib.HSS_ERR_QUERY:
            check(rc)
        return rc

    def last_status(self, n):
        st = np.zeros(max(n, 1), np.int32)
        check(_lib.load().hss_searcher_last_status(self._h, _np_ptr(st), n))
        return st[:n]

    def last_candidates(self, query, cap=1 << 20):
        """(approximate scores, locations, count, theta, eps) of one query of the last batch."""
        sc = np.zeros(cap, np.float32)
        loc = np.zeros(cap, np.uint32)
        n, th, ep = ctypes.c_uint32(), ctypes.c_float(), ctypes.c_float()
        check(_lib.load().hss_searcher_last_candidates(self._h, query, _np_ptr(sc), _np_ptr(loc), cap,
                                                       ctypes.byref(n), ctypes.byref(th), ctypes.byref(ep)))
        k = min(n.value, cap)
        return sc[:k], loc[:k], n.value, th.value, ep.value

    def feature_dim(self):
        return _lib.load().hss_searcher_feature_dim(self._h)

    def features(self, d_queries, nq, filters, topks, d_x, stream=0):
        """Feature rows [nq][feature_dim] of a batch into device memory d_x (runs the filter stage and
        the doc sample)."""
        t = np.ascontiguousarray(topks, dtype=np.uint32)
        check(_lib.load().hss_searcher_features(self._h, d_queries, nq, filters._h, _np_ptr(t), d_x, stream))

    def set_threshold_model(self, model, margin):
        """Learned threshold on (model) or off (None); margin is subtracted from the prediction."""
        check(_lib.load().hss_searcher_set_threshold_model(self._h, model._h if model else None, margin))
        self._model = model  # kept alive while the searcher uses it

    def last_thresholds(self, n):
        """(doc sample's proven thresholds, the thresholds the model set) of the last batch."""
        t1 = np.zeros(max(n, 1), np.float32)
        ta = np.zeros(max(n, 1), np.float32)
        check(_lib.load().hss_searcher_last_thresholds(self._h, _np_ptr(t1), _np_ptr(ta), n))
        return t1[:n], ta[:n]

    def last_candidate_counts(self, n):
        """Docs that cleared each query's threshold in its last candidate pass of the last batch."""
        c = np.zeros(max(n, 1), np.uint32)
        check(_lib.load().hss_searcher_last_candidate_counts(self._h, _np_ptr(c), n))
        return c[:n]

    def last_threshold_misses(self, n):
        """Per query of the last batch: True where the model's threshold was too high and the query was
        re-run at a proven threshold."""
        m = np.zeros(max(n, 1), np.uint8)
        check(_lib.load().hss_searcher_last_threshold_misses(self._h, _np_ptr(m), n))
        return m[:n].astype(bool)

    def set_pipeline_test(self, hold_load, wait_budget_cycles=0):
        """The next batch's first single-SM tensor-core pass withholds its hold_load-th corpus load
        (hss_searcher_set_pipeline_test): its bounded wait runs out and the batch reports the error."""
        check(_lib.load().hss_searcher_set_pipeline_test(self._h, hold_load, wait_budget_cycles))

    def set_timing(self, on=True):
        check(_lib.load().hss_searcher_set_timing(self._h, int(on)))

    def set_graphs(self, on=True):
        """CUDA-graph replay per batch shape (hss_searcher_set_graphs): query and output buffers of
        maxBatch rows."""
        check(_lib.load().hss_searcher_set_graphs(self._h, int(on)))

    def graph_stats(self):
        c, r, ms, f = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_double(), ctypes.c_int32()
        check(_lib.load().hss_searcher_graph_stats(self._h, ctypes.byref(c), ctypes.byref(r), ctypes.byref(ms),
                                                   ctypes.byref(f)))
        return {"captures": c.value, "replays": r.value, "failed": bool(f.value), "capture_ms": ms.value}

    def last_times(self):
        ms = np.zeros(5, np.float32)
        r, l = ctypes.c_uint32(), ctypes.c_uint32()
        check(_lib.load().hss_searcher_last_times(self._h, _np_ptr(ms), ctypes.byref(r), ctypes.byref(l)))
        return {"filter_ms": float(ms[0]), "sample_ms": float(ms[1]), "candidates_ms": float(ms[2]),
                "select_ms": float(ms[3]), "total_ms": float(ms[4]), "retries": r.value, "launches": l.value}


class Server:
    """The serving loop (continuous batching over one resident table; include/hss.h, hss_server_*)."""

    def __init__(self, table, slots=2, max_batch=256, max_wait_us=200, method=0, memory_budget=0, candidate_cap=0,
                 sample_docs=0, graphs=False):
        cfg = _lib.ServerConfig(slots, max_batch, max_wait_us, method, memory_budget, candidate_cap, sample_docs,
                                1 if graphs else 0)
        h = ctypes.c_void_p()
        check(_lib.load().hss_server_create(table._h, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.table = table
        self.dim = table.info["dim"]

    def close(self):
        if self._h:
            _lib.load().hss_server_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, filter_expr, vector, topk):
        v = np.ascontiguousarray(vector, dtype=np.float32)
        rid = ctypes.c_uint64()
        check(_lib.load().hss_server_submit(self._h, _np_ptr(v), v.size, (filter_expr or "").encode(), topk,
                                            ctypes.byref(rid)))
        return rid.value

    def wait(self, rid, cap=_lib.HSS_MAX_TOPK, timeout_ms=-1):
        """(scores, ids, latency ms, status) of request rid, or None on timeout."""
        sc = np.zeros(max(cap, 1), np.float32)
        ids = np.zeros(max(cap, 1), np.int64)
        n, lat, st = ctypes.c_uint32(), ctypes.c_double(), ctypes.c_int32()
        rc = _lib.load().hss_server_wait(self._h, rid, _np_ptr(sc), _np_ptr(ids), cap, ctypes.byref(n),
                                         ctypes.byref(lat), ctypes.byref(st), timeout_ms)
        if rc == 1:
            return None
        check(rc)
        k = min(n.value, cap)
        return sc[:k], ids[:k], lat.value, st.value

    def stats(self):
        st = _lib.ServerStats()
        check(_lib.load().hss_server_get_stats(self._h, ctypes.byref(st)))
        return {"completed": st.completed, "batches": st.batches, "slots": st.slots, "mean_batch": st.meanBatch,
                "p50_ms": st.p50Ms, "p99_ms": st.p99Ms, "max_ms": st.maxMs, "graph_captures": st.graphCaptures,
                "graph_replays": st.graphReplays, "graph_capture_ms": st.graphCaptureMs}

    def reset_stats(self):
        check(_lib.load().hss_server_reset_stats(self._h))

    def set_threshold_model(self, model, margin):
        check(_lib.load().hss_server_set_threshold_model(self._h, model._h if model else None, margin))
        self._model = model

    def run_poisson(self, queries, exprs, topks, rate_qps, seed=0):
        """Open-loop Poisson arrivals at rate_qps; returns (latencies ms [n], offered QPS, wall seconds)."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        n = len(q)
        arr = (ctypes.c_char_p * max(n, 1))(*[(e or "").encode() for e in exprs])
        t = np.ascontiguousarray(topks, dtype=np.uint32)
        lat = np.zeros(max(n, 1), np.float64)
        offered, wall = ctypes.c_double(), ctypes.c_double()
        check(_lib.load().hss_server_run_poisson(self._h, _np_ptr(q), n, arr, _np_ptr(t), float(rate_qps), seed,
                                                 _np_ptr(lat), ctypes.byref(offered), ctypes.byref(wall)))
        return lat[:n], offered.value, wall.value


class ThresholdModel:
    """The learned K-th-score predictor (MLP din -> hidden -> hidden -> 1, GELU) on one GPU. Parameters
    are one flat FP32 vector: W1 [din][hidden], b1, W2 [hidden][hidden], b2, w3 [hidden], b3."""

    def __init__(self, din, hidden=256, device=0, seed=0):
        h = ctypes.c_void_p()
        check(_lib.load().hss_model_create(device, din, hidden, seed, ctypes.byref(h)))
        self._h = h
        self.din, self.hidden, self.device = din, hidden, device
        self.scale, self.shift = 1.0, 0.0

    def close(self):
        if self._h:
            _lib.load().hss_model_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def param_count(self):
        return _lib.load().hss_model_param_count(self._h)

    def get_params(self):
        p = np.zeros(self.param_count, np.float32)
        check(_lib.load().hss_model_get_params(self._h, _np_ptr(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.param_count
        check(_lib.load().hss_model_set_params(self._h, _np_ptr(p)))

    def set_output_scale(self, scale, shift):
        self.scale, self.shift = float(scale), float(shift)
        check(_lib.load().hss_model_set_output_scale(self._h, self.scale, self.shift))

    def set_quantile(self, tau):
        """Training loss: 0 the mean squared error; tau in (0, 1) the pinball loss of the tau-quantile."""
        check(_lib.load().hss_model_set_quantile(self._h, float(tau)))

    def forward(self, d_x, batch, d_y, stream=0):
        check(_lib.load().hss_model_forward(self._h, d_x, batch, d_y, stream))

    def train_step(self, d_x, d_t, batch, lr, stream=0):
        loss = ctypes.c_float()
        check(_lib.load().hss_model_train_step(self._h, d_x, d_t, batch, lr, ctypes.byref(loss), stream))
        return loss.value

    def gradients(self, d_x, d_t, batch, stream=0):
        g = np.zeros(self.param_count, np.float32)
        loss = ctypes.c_float()
        check(_lib.load().hss_model_gradients(self._h, d_x, d_t, batch, _np_ptr(g), ctypes.byref(loss), stream))
        return g, loss.value


# ---- operator entry points (device pointers as ints) ----

def vector_score(d_queries, d_docs, d_out, m, n, k, ld, stream=0):
    check(_lib.load().hss_vector_score_launch(d_queries, d_docs, d_out, m, n, k, ld, stream))


def bitmap_text_filter(d_postings, d_expr, context, d_result, d_status=None, stream=0):
    check(_lib.load().hss_bitmap_text_filter_launch(d_postings, d_expr, None, context, d_result, d_status, stream))


def posting_bitlist_to_set(d_postings, byte_size, d_results, count, d_status=None, stream=0):
    check(_lib.load().hss_posting_bitlist_to_set_launch(d_postings, byte_size, d_results, count, d_status, stream))


def aggregator_workspace_size(doc_number):
    return _lib.load().hss_aggregator_workspace_size(doc_number)


def aggregator(d_filter, d_scores, d_loc, d_out_scores, d_out_loc, d_count, doc_number, d_ws, ws_bytes, stream=0):
    check(_lib.load().hss_aggregator_launch(d_filter, d_scores, d_loc, d_out_scores, d_out_loc, d_count, doc_number,
                                            d_ws, ws_bytes, stream))


def aggregator_noalloc(d_filter, d_scores, d_loc, d_out_scores, d_out_loc, d_count, doc_number, stream=0):
    """hss_aggregator_launch_noalloc: the aggregator with its scratch compiled into the library (no
    workspace, no allocation; doc_number <= HSS_AGGREGATOR_NOALLOC_MAX_DOCS; calls on one device must
    not overlap on the GPU)."""
    check(_lib.load().hss_aggregator_launch_noalloc(d_filter, d_scores, d_loc, d_out_scores, d_out_loc, d_count,
                                                    doc_number, stream))


def topk(d_scores, d_locs, d_count, k, d_out_scores, d_out_locs, d_out_count, stream=0):
    check(_lib.load().hss_topk_launch(d_scores, d_locs, d_count, k, d_out_scores, d_out_locs, d_out_count, stream))


def merge_shards(d_scores, d_ids, d_counts, nq, in_stride, k, d_out_scores, d_out_ids, d_out_counts, out_stride,
                 stream=0):
    """hss_merge_shards_launch: per-shard sorted results (lists of device pointers) merged into the
    global top-k on the device."""
    n = len(d_scores)
    arr = lambda xs: (ctypes.c_void_p * n)(*xs)
    check(_lib.load().hss_merge_shards_launch(arr(d_scores), arr(d_ids), arr(d_counts), n, nq, in_stride, k,
                                              d_out_scores, d_out_ids, d_out_counts, out_stride, stream))


def hash64(token):
    b = token.encode() if isinstance(token, str) else bytes(token)
    return _lib.load().hss_hash64(b, len(b))


def posting_serialize(ids, doc_num, is_matrix=False, density_threshold=1.0 / 64, sparse_packed=False):
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    cap = 8 + max(doc_num, 6 * ((doc_num + 15) // 16), 4 * ids.size) + 64
    out = np.zeros(cap, np.uint8)
    n = check(_lib.load().hss_posting_serialize(_np_ptr(ids), ids.size, doc_num, int(is_matrix), density_threshold,
                                                int(sparse_packed), _np_ptr(out), cap))
    return out[:n].tobytes()


def device_count():
    return _lib.load().hss_device_count()
