"""ctypes binding of libhss.so (the C-ABI declared in include/hss.h).

The library is built in-tree by ``__graft_entry__.build()`` (``make -C hybridsearchsystem_b200/csrc``).
Loading fails loudly when it is missing: there is no CPU fallback for any operation.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhss.so")

c_f32p = ctypes.POINTER(ctypes.c_float)
c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_i32p = ctypes.POINTER(ctypes.c_int32)
c_i64p = ctypes.POINTER(ctypes.c_int64)
c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_u8p = ctypes.POINTER(ctypes.c_uint8)
vp = ctypes.c_void_p

HSS_OK = 0
HSS_ERR_INVALID = -1
HSS_ERR_CUDA = -2
HSS_ERR_PARSE = -3
HSS_ERR_PROGRAM = -4
HSS_ERR_LIMIT = -5
HSS_ERR_INDEX = -6
HSS_ERR_QUERY = -7

HSS_MAX_TOPK = 4096
HSS_AGGREGATOR_NOALLOC_MAX_DOCS = 16777216
HSS_MAX_OPERANDS = 64
HSS_MAX_PROGRAM = 512
HSS_FILTER_HEAD_ADDRESSES = 0x80000000

QSTATUS_BAD_PROGRAM = 1
QSTATUS_BAD_POSTING = 2
QSTATUS_OVERFLOW = 4
QSTATUS_TOPK_TOO_LARGE = 8


class HssError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libhss error {code}: {msg}")
        self.code = code


class FilterContext(ctypes.Structure):
    """TextFilterContextData (device_common_external.h:17-25)."""

    _fields_ = [(n, ctypes.c_uint32) for n in
                ("postingNum", "segmentNum", "segmentLength", "tileNum", "exprLen", "opNum", "flags")]


class IndexConfig(ctypes.Structure):
    _fields_ = [("docNumPerSegment", ctypes.c_uint32), ("densityThreshold", ctypes.c_float),
                ("matrixPosting", ctypes.c_int32), ("sparsePacked", ctypes.c_int32),
                ("docOffset", ctypes.c_uint64)]


class SearcherConfig(ctypes.Structure):
    _fields_ = [("maxBatch", ctypes.c_uint32), ("candidateCap", ctypes.c_uint32),
                ("sampleDocs", ctypes.c_uint32), ("maxRetries", ctypes.c_uint32), ("method", ctypes.c_int32),
                ("decodeInPlace", ctypes.c_int32)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_uint32), ("maxBatch", ctypes.c_uint32), ("maxWaitUs", ctypes.c_uint32),
                ("method", ctypes.c_int32), ("memoryBudget", ctypes.c_uint64), ("candidateCap", ctypes.c_uint32),
                ("sampleDocs", ctypes.c_uint32), ("graphs", ctypes.c_uint32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("batches", ctypes.c_uint64), ("slots", ctypes.c_uint32),
                ("meanBatch", ctypes.c_double), ("p50Ms", ctypes.c_double), ("p99Ms", ctypes.c_double),
                ("maxMs", ctypes.c_double), ("graphCaptures", ctypes.c_uint64), ("graphReplays", ctypes.c_uint64),
                ("graphCaptureMs", ctypes.c_double)]


# (name, restype, argtypes) for every symbol include/hss.h declares.
SIGNATURES = [
    ("hss_vector_score_launch", ctypes.c_int,
     [vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, vp]),
    ("hss_bitmap_text_filter_launch", ctypes.c_int, [vp, vp, vp, FilterContext, vp, vp, vp]),
    ("hss_posting_bitlist_to_set_launch", ctypes.c_int, [vp, ctypes.c_uint32, vp, ctypes.c_uint32, vp, vp]),
    ("hss_aggregator_workspace_size", ctypes.c_size_t, [ctypes.c_uint32]),
    ("hss_aggregator_launch", ctypes.c_int,
     [vp, vp, vp, vp, vp, vp, ctypes.c_uint32, vp, ctypes.c_size_t, vp]),
    ("hss_aggregator_launch_noalloc", ctypes.c_int, [vp, vp, vp, vp, vp, vp, ctypes.c_uint32, vp]),
    ("hss_topk_launch", ctypes.c_int, [vp, vp, vp, ctypes.c_uint32, vp, vp, vp, vp]),
    ("hss_merge_shards_launch", ctypes.c_int,
     [vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, vp, vp, vp, ctypes.c_uint32,
      vp]),
    ("hss_table_build", ctypes.c_int,
     [ctypes.c_int32, vp, vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
      ctypes.POINTER(IndexConfig), ctypes.POINTER(vp)]),
    ("hss_table_build_device", ctypes.c_int,
     [ctypes.c_int32, vp, vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
      ctypes.POINTER(IndexConfig), ctypes.POINTER(vp)]),
    ("hss_table_load", ctypes.c_int, [ctypes.c_int32, ctypes.c_char_p, ctypes.POINTER(vp)]),
    ("hss_table_save", ctypes.c_int, [vp, ctypes.c_char_p]),
    ("hss_table_load_reference", ctypes.c_int, [ctypes.c_int32, ctypes.c_char_p, ctypes.POINTER(vp)]),
    ("hss_table_save_reference", ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_uint32]),
    ("hss_table_load_times", ctypes.c_int, [vp, vp, c_u64p, c_u64p, c_u32p]),
    ("hss_table_free", None, [vp]),
    ("hss_table_info", ctypes.c_int, [vp, c_u64p, c_u32p, c_u32p, c_u32p, c_u32p, c_f32p]),
    ("hss_table_posting", ctypes.c_int,
     [vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(c_u8p), c_u32p]),
    ("hss_table_device_ptrs", ctypes.c_int, [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp)]),
    ("hss_searcher_create", ctypes.c_int, [vp, ctypes.POINTER(SearcherConfig), ctypes.POINTER(vp)]),
    ("hss_searcher_workspace_bytes", ctypes.c_size_t, [vp, ctypes.POINTER(SearcherConfig)]),
    ("hss_table_prepare", ctypes.c_int, [vp, ctypes.POINTER(SearcherConfig)]),
    ("hss_searcher_create_in", ctypes.c_int,
     [vp, ctypes.POINTER(SearcherConfig), vp, ctypes.c_size_t, ctypes.POINTER(vp)]),
    ("hss_searcher_free", None, [vp]),
    ("hss_searcher_add_query", ctypes.c_int, [vp, ctypes.c_char_p, vp, ctypes.c_uint32, ctypes.c_uint32]),
    ("hss_searcher_batch_search", ctypes.c_int, [vp, vp, vp, vp, ctypes.c_uint32]),
    ("hss_filters_compile", ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_char_p), ctypes.c_uint32, ctypes.POINTER(vp)]),
    ("hss_filters_free", None, [vp]),
    ("hss_searcher_search_device", ctypes.c_int,
     [vp, vp, ctypes.c_uint32, vp, vp, vp, vp, vp, ctypes.c_uint32, vp]),
    ("hss_searcher_search_device_async", ctypes.c_int,
     [vp, vp, ctypes.c_uint32, vp, vp, vp, vp, vp, ctypes.c_uint32, vp]),
    ("hss_searcher_finish", ctypes.c_int, [vp]),
    ("hss_searcher_filter_device", ctypes.c_int, [vp, vp, ctypes.c_uint32, vp, ctypes.c_uint64, vp, vp]),
    ("hss_searcher_last_status", ctypes.c_int, [vp, vp, ctypes.c_uint32]),
    ("hss_searcher_last_candidates", ctypes.c_int,
     [vp, ctypes.c_uint32, vp, vp, ctypes.c_uint32, c_u32p, c_f32p, c_f32p]),
    ("hss_searcher_set_pipeline_test", ctypes.c_int, [vp, ctypes.c_uint32, ctypes.c_uint64]),
    ("hss_searcher_set_timing", ctypes.c_int, [vp, ctypes.c_int32]),
    ("hss_searcher_last_times", ctypes.c_int, [vp, vp, c_u32p, c_u32p]),
    ("hss_searcher_set_graphs", ctypes.c_int, [vp, ctypes.c_int32]),
    ("hss_searcher_graph_stats", ctypes.c_int, [vp, vp, vp, vp, c_i32p]),
    ("hss_hash64", ctypes.c_uint64, [ctypes.c_char_p, ctypes.c_uint32]),
    ("hss_posting_serialize", ctypes.c_int64,
     [vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int32, ctypes.c_float, ctypes.c_int32, vp, ctypes.c_uint64]),
    ("hss_filter_compile", ctypes.c_int,
     [vp, ctypes.c_char_p, vp, ctypes.c_uint32, c_u32p, vp, ctypes.c_uint32, c_u32p, c_u32p, c_i32p]),
    ("hss_searcher_feature_dim", ctypes.c_uint32, [vp]),
    ("hss_searcher_features", ctypes.c_int, [vp, vp, ctypes.c_uint32, vp, vp, vp, vp]),
    ("hss_searcher_set_threshold_model", ctypes.c_int, [vp, vp, ctypes.c_float]),
    ("hss_searcher_last_thresholds", ctypes.c_int, [vp, vp, vp, ctypes.c_uint32]),
    ("hss_searcher_last_candidate_counts", ctypes.c_int, [vp, vp, ctypes.c_uint32]),
    ("hss_searcher_last_threshold_misses", ctypes.c_int, [vp, vp, ctypes.c_uint32]),
    ("hss_model_create", ctypes.c_int, [ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                        ctypes.POINTER(vp)]),
    ("hss_model_free", None, [vp]),
    ("hss_model_param_count", ctypes.c_uint64, [vp]),
    ("hss_model_get_params", ctypes.c_int, [vp, vp]),
    ("hss_model_set_params", ctypes.c_int, [vp, vp]),
    ("hss_model_set_output_scale", ctypes.c_int, [vp, ctypes.c_float, ctypes.c_float]),
    ("hss_model_set_quantile", ctypes.c_int, [vp, ctypes.c_float]),
    ("hss_model_forward", ctypes.c_int, [vp, vp, ctypes.c_uint32, vp, vp]),
    ("hss_model_train_step", ctypes.c_int, [vp, vp, vp, ctypes.c_uint32, ctypes.c_float,
                                            ctypes.POINTER(ctypes.c_float), vp]),
    ("hss_model_gradients", ctypes.c_int, [vp, vp, vp, ctypes.c_uint32, vp, ctypes.POINTER(ctypes.c_float), vp]),
    ("hss_server_create", ctypes.c_int, [vp, ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]),
    ("hss_server_free", None, [vp]),
    ("hss_server_submit", ctypes.c_int, [vp, vp, ctypes.c_uint32, ctypes.c_char_p, ctypes.c_uint32,
                                         ctypes.POINTER(ctypes.c_uint64)]),
    ("hss_server_wait", ctypes.c_int, [vp, ctypes.c_uint64, vp, vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32),
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32),
                                       ctypes.c_int32]),
    ("hss_server_get_stats", ctypes.c_int, [vp, ctypes.POINTER(ServerStats)]),
    ("hss_server_reset_stats", ctypes.c_int, [vp]),
    ("hss_server_set_threshold_model", ctypes.c_int, [vp, vp, ctypes.c_float]),
    ("hss_server_run_poisson", ctypes.c_int, [vp, vp, ctypes.c_uint32, vp, vp, ctypes.c_double, ctypes.c_uint64, vp,
                                              ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    ("hss_last_error", ctypes.c_char_p, []),
    ("hss_device_count", ctypes.c_int, []),
]

_lib = None


def load():
    """Loads libhss.so (once) and binds every C-ABI symbol. Raises if the library is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise HssError(HSS_ERR_INVALID, f"{LIB_PATH} not built; run __graft_entry__.build()")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc):
    """Raises HssError for a negative status code."""
    if rc < 0:
        msg = load().hss_last_error()
        raise HssError(rc, msg.decode() if msg else "")
    return rc
