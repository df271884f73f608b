"""B200-native filtered full-recall search: the reference's single-batch filtered full-recall path
(posting filter -> exact inner-product scoring -> top-K) as hand-written sm_100a CUDA behind a
C-ABI (include/hss.h, libhss.so) with a host C++ mirror of the reference's DataTable /
FullRecallSearcher / QueryNode interface.
"""
from . import data
from ._lib import HssError, load
from .api import (DataTable, Filters, FullRecallSearcher, Server, ThresholdModel, aggregator, aggregator_noalloc, aggregator_workspace_size,
                  bitmap_text_filter, device_count, hash64, merge_shards, posting_bitlist_to_set, posting_serialize, topk,
                  vector_score)

__all__ = ["DataTable", "Filters", "FullRecallSearcher", "HssError", "Server", "ThresholdModel", "aggregator", "aggregator_noalloc",
           "aggregator_workspace_size",
           "bitmap_text_filter", "data", "device_count", "hash64", "load", "merge_shards", "posting_bitlist_to_set",
           "posting_serialize", "topk", "vector_score"]
