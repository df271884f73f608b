"""Python access to the oracle -- TEST INFRASTRUCTURE ONLY.

`oracle` wraps liboracle.so, the C restatement of the reference's CPU path (oracle.c), and `ref` wraps
_ref/libref.so, the reference's own CPU code compiled from its sources (ref_shim.cpp). Only the tests,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this package, and only as the
checker; the product (hybridsearchsystem_b200) never does.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")

vp = ctypes.c_void_p


class Node(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int32), ("nkids", ctypes.c_int32), ("kid0", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("tag", ctypes.c_uint64)]


_o = None
_r = None


def lib():
    global _o
    if _o is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"{ORACLE_SO} missing: run `make -C oracle`")
        o = ctypes.CDLL(ORACLE_SO)
        o.orc_parse.argtypes = [ctypes.c_char_p, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        o.orc_parse.restype = ctypes.c_int
        o.orc_eval_bitmap.argtypes = [vp, vp, ctypes.c_int, vp, ctypes.c_uint32]
        o.orc_eval_bitmap.restype = ctypes.c_int
        o.orc_filter_bits.argtypes = [vp, vp, ctypes.c_int, vp, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, vp]
        o.orc_filter_bits.restype = None
        o.orc_topk_batch.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp, vp, vp, vp, vp, ctypes.c_uint32,
                                     ctypes.c_uint64, ctypes.c_uint64, vp, ctypes.c_int32, vp, vp, vp, ctypes.c_int]
        o.orc_topk_batch.restype = None
        o.orc_score_f64.argtypes = [vp, ctypes.c_uint32, vp, vp, ctypes.c_int, vp]
        o.orc_score_f64.restype = None
        o.orc_posting_serialize.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.c_float,
                                            ctypes.c_int, vp, ctypes.c_uint64]
        o.orc_posting_serialize.restype = ctypes.c_int64
        o.orc_posting_decode.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint32, vp]
        o.orc_posting_decode.restype = ctypes.c_int
        o.orc_eval_postfix.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp, ctypes.c_uint32, ctypes.c_uint32, vp]
        o.orc_eval_postfix.restype = ctypes.c_int
        o.orc_hash64.argtypes = [ctypes.c_char_p, ctypes.c_uint32]
        o.orc_hash64.restype = ctypes.c_uint64
        _o = o
    return _o


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    """The reference's own CPU code (raises when _ref/libref.so was not built)."""
    global _r
    if _r is None:
        os.environ.setdefault("NPUR_LOG_LEVEL", "ERROR")
        r = ctypes.CDLL(REF_SO)
        r.ref_hash64.argtypes = [ctypes.c_char_p, ctypes.c_uint32]
        r.ref_hash64.restype = ctypes.c_uint64
        r.ref_posting_serialize.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.c_float, vp,
                                            ctypes.c_uint64]
        r.ref_posting_serialize.restype = ctypes.c_int64
        r.ref_parse_ok.argtypes = [ctypes.c_char_p]
        r.ref_parse_ok.restype = ctypes.c_int
        r.ref_eval_bitmap.argtypes = [ctypes.c_char_p, vp, ctypes.c_uint32]
        r.ref_eval_bitmap.restype = ctypes.c_int
        r.ref_cpu_topk.argtypes = [vp, ctypes.c_uint32, ctypes.c_char_p, vp, vp, ctypes.c_uint32, ctypes.c_uint64,
                                   ctypes.c_uint64, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int]
        r.ref_cpu_topk.restype = ctypes.c_int
        r.ref_cpu_topk_batch.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_char_p), vp, vp,
                                         vp, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int32, vp, vp]
        r.ref_cpu_topk_batch.restype = ctypes.c_int
        r.ref_f32_to_f16.argtypes = [ctypes.c_float]
        r.ref_f32_to_f16.restype = ctypes.c_uint16
        r.ref_f16_to_f32.argtypes = [ctypes.c_uint16]
        r.ref_f16_to_f32.restype = ctypes.c_float
        _r = r
    return _r


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


class Parsed:
    """A filter parsed by the restated grammar (root < 0: match all)."""

    def __init__(self, expr, cap=4096):
        self.nodes = (Node * cap)()
        self.kids = np.zeros(cap, np.int32)
        root = ctypes.c_int(-1)
        rc = lib().orc_parse(expr.encode(), self.nodes, cap, _p(self.kids), cap, ctypes.byref(root))
        self.ok = rc >= 0
        self.root = root.value
        self.count = max(rc, 0)


def parse_ok(expr):
    return Parsed(expr).ok


def eval_bitmap(expr, bm):
    p = Parsed(expr)
    if not p.ok:
        return -1
    bm = np.ascontiguousarray(bm, np.uint64)
    return lib().orc_eval_bitmap(p.nodes, _p(p.kids), p.root, _p(bm), bm.size)


def filter_bits(expr, bits, doc_num=None, doc_offset=0):
    """Packed per-doc filter result (bit i%64 of word i/64) over docs [doc_offset, doc_offset+doc_num)."""
    p = Parsed(expr)
    if not p.ok:
        raise ValueError(f"filter does not parse: {expr!r}")
    bits = np.ascontiguousarray(bits, np.uint64)
    n = bits.shape[0] - doc_offset if doc_num is None else doc_num
    out = np.zeros((n + 63) // 64, np.uint64)
    lib().orc_filter_bits(p.nodes, _p(p.kids), p.root, _p(bits), bits.shape[1], n, doc_offset, _p(out))
    return out


def topk(queries, exprs, topks, vectors, bits, threads=1, doc_offset=0, doc_num=None, out_stride=None):
    """Ordered ground truth: (scores [nq][stride], ids [nq][stride], counts [nq]), (score desc, id asc)."""
    queries = np.ascontiguousarray(queries, np.float32)
    vectors = np.ascontiguousarray(vectors, np.float32)
    bits = np.ascontiguousarray(bits, np.uint64)
    nq, dim = queries.shape
    topks = np.ascontiguousarray(np.broadcast_to(np.asarray(topks, np.int32), (nq,)), np.int32)
    stride = out_stride or max(1, int(topks.max(initial=1)))
    cap = 64 * nq + 4096
    nodes = (Node * cap)()
    kids = np.zeros(cap, np.int32)
    roots = np.zeros(nq, np.int32)
    used_n = used_k = 0
    for i, e in enumerate(exprs):
        sub_nodes = (Node * 4096)()
        sub_kids = np.zeros(4096, np.int32)
        root = ctypes.c_int(-1)
        rc = lib().orc_parse(e.encode(), sub_nodes, 4096, _p(sub_kids), 4096, ctypes.byref(root))
        if rc < 0:
            raise ValueError(f"filter does not parse: {e!r}")
        if used_n + rc > cap or used_k + rc > cap:
            raise ValueError("filters too large for the batch oracle")
        nk = sum(sub_nodes[j].nkids for j in range(rc))
        for j in range(rc):
            nd = sub_nodes[j]
            nodes[used_n + j] = Node(nd.op, nd.nkids, nd.kid0 + used_k, 0, nd.tag)
        kids[used_k:used_k + nk] = sub_kids[:nk] + used_n
        roots[i] = root.value + used_n if root.value >= 0 else -1
        used_n += rc
        used_k += nk
    n = vectors.shape[0] - doc_offset if doc_num is None else doc_num
    scores = np.zeros((nq, stride), np.float32)
    ids = np.full((nq, stride), -1, np.int64)
    counts = np.zeros(nq, np.int32)
    lib().orc_topk_batch(_p(queries), nq, dim, nodes, _p(kids), _p(roots), _p(vectors), _p(bits), bits.shape[1],
                         n, doc_offset, _p(topks), stride, _p(scores), _p(ids), _p(counts), threads)
    return scores, ids, counts


def score_f64(query, vectors, ids):
    query = np.ascontiguousarray(query, np.float32)
    ids = np.ascontiguousarray(ids, np.int64)
    out = np.zeros(ids.size, np.float64)
    lib().orc_score_f64(_p(query), query.size, _p(np.ascontiguousarray(vectors, np.float32)), _p(ids), ids.size,
                        _p(out))
    return out


def posting_serialize(ids, seg_docs, is_matrix=False, threshold=1.0 / 64, packed=False):
    ids = np.ascontiguousarray(ids, np.uint32)
    cap = 8 + max(seg_docs, 6 * ((seg_docs + 15) // 16), 4 * ids.size) + 64
    out = np.zeros(cap, np.uint8)
    n = lib().orc_posting_serialize(_p(ids), ids.size, seg_docs, int(is_matrix), threshold, int(packed), _p(out), cap)
    if n < 0:
        raise ValueError("posting cannot be serialised")
    return out[:n].tobytes()


def posting_decode(posting, seg_docs):
    buf = np.frombuffer(posting, np.uint8).copy()
    out = np.zeros((seg_docs + 63) // 64, np.uint64)
    layout = lib().orc_posting_decode(_p(buf), buf.size, seg_docs, _p(out))
    return layout, out


def eval_postfix(prog, op_count, operands, words):
    """Evaluates a postfix program over dense operand bitsets (each `words` u64). None if malformed."""
    prog = np.ascontiguousarray(prog, np.uint32)
    ops = [np.ascontiguousarray(o, np.uint64) for o in operands]
    arr = (ctypes.c_void_p * max(1, len(ops)))(*[o.ctypes.data for o in ops])
    out = np.zeros(words, np.uint64)
    rc = lib().orc_eval_postfix(_p(prog), prog.size, op_count, arr, len(ops), words, _p(out))
    return None if rc != 0 else out


def hash64(token):
    b = token.encode() if isinstance(token, str) else bytes(token)
    return lib().orc_hash64(b, len(b))
