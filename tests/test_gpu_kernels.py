"""Operator-level parity on the GPU, through the C-ABI: the batched posting filter and the
BitmapTextFilter / PostingBitListToSet / kernel_vector_mmad / Aggregator / TOPK drop-ins, each against
the oracle on the same seeded inputs. Integer and index outputs must match bit for bit; the exact
scorer must reproduce the ground truth's FP32 scores bit for bit."""
import numpy as np
import pytest

import hybridsearchsystem_b200 as hss
import oracle
from hybridsearchsystem_b200 import _lib, data

pytestmark = pytest.mark.gpu


def _table(torch, layout="bitmap", n=5000, tags=96, p=1024, seed=3, dim=32):
    kw = {"bitmap": {}, "packed": {"sparse_packed": True}, "matrix": {"matrix_posting": True}}[layout]
    mix = data.Mixture(dim, tags, (0.002, 0.6), n_clusters=16, seed=seed)
    vec, bits, _ = mix.corpus(n, seed=seed + 100)
    table = hss.DataTable.build(vec, bits, tags, device=0, doc_num_per_segment=p, **kw)
    return mix, vec, bits, table


def _edge_filters():
    return ["", "5", "NOT 5", "NOT NOT 7", "1 AND 1", "200 OR 3", "NOT 250", "3 AND NOT 3", "250",
            "(1 OR 2) AND (3 OR 4)", "NOT (1 OR 2 OR 3 OR 4 OR 5 OR 6)", "0 OR 95", "NOT 0 AND NOT 95"]


def _bits_of(words, n):
    return np.unpackbits(np.ascontiguousarray(words).view(np.uint8), bitorder="little")[:n]


@pytest.mark.parametrize("in_place", [False, True], ids=["dense_matrix", "in_place"])
@pytest.mark.parametrize("layout", ["bitmap", "packed", "matrix"])
def test_batched_filter_matches_oracle(torch_cuda, layout, in_place):
    torch = torch_cuda
    mix, vec, bits, table = _table(torch, layout)
    info = table.info
    exprs = data.make_filters(mix, 60, n_tags=(1, 6), seed=9) + _edge_filters()
    s = hss.FullRecallSearcher(table, max_batch=len(exprs), candidate_cap=4096, decode_in_place=in_place)
    f = s.compile_filters(exprs)
    words = info["segment_num"] * info["doc_num_per_segment"] // 64
    out = torch.zeros((len(exprs), words), dtype=torch.int64, device="cuda")
    cnt = torch.zeros(len(exprs), dtype=torch.int32, device="cuda")
    assert s.filter_device(f, len(exprs), out.data_ptr(), words, cnt.data_ptr()) == _lib.HSS_OK
    got = out.cpu().numpy().view(np.uint64)
    counts = cnt.cpu().numpy()
    n = vec.shape[0]
    for i, e in enumerate(exprs):
        want = _bits_of(oracle.filter_bits(e, bits), n)
        row = _bits_of(got[i], words * 64)
        assert (row[:n] == want).all(), e
        assert not row[n:].any(), e  # docs past docNum are cleared
        assert counts[i] == want.sum(), e


@pytest.mark.parametrize("in_place", [False, True], ids=["dense_matrix", "in_place"])
def test_batched_filter_wide_segments_six_operands(torch_cuda, in_place):
    # 131072-doc segments and six-operand programs: the widest per-thread word counts and the largest
    # operand slots in shared memory (48 KB next to the program)
    torch = torch_cuda
    mix = data.Mixture(32, 64, (1e-3, 0.5), n_clusters=16, seed=61)
    vec, bits, _ = mix.corpus(140000, seed=62)
    table = hss.DataTable.build(vec, bits, 64, device=0, doc_num_per_segment=131072)
    info = table.info
    rng = np.random.default_rng(63)
    exprs = []
    for i in range(40):
        t = rng.choice(64, 6, replace=False)
        ops = rng.choice(["AND", "OR"], 5)
        e = str(t[0])
        for o, x in zip(ops, t[1:]):
            e = f"({e} {o} {'NOT ' if rng.random() < 0.3 else ''}{x})"
        exprs.append(e)
    s = hss.FullRecallSearcher(table, max_batch=len(exprs), candidate_cap=4096, decode_in_place=in_place)
    f = s.compile_filters(exprs)
    words = info["segment_num"] * info["doc_num_per_segment"] // 64
    out = torch.zeros((len(exprs), words), dtype=torch.int64, device="cuda")
    cnt = torch.zeros(len(exprs), dtype=torch.int32, device="cuda")
    assert s.filter_device(f, len(exprs), out.data_ptr(), words, cnt.data_ptr()) == _lib.HSS_OK
    got = out.cpu().numpy().view(np.uint64)
    n = vec.shape[0]
    for i, e in enumerate(exprs):
        want = _bits_of(oracle.filter_bits(e, bits), n)
        row = _bits_of(got[i], words * 64)
        assert (row[:n] == want).all(), e
        assert not row[n:].any(), e
        assert int(cnt.cpu().numpy()[i]) == want.sum(), e


# The dense filter's CTAs take 4, 2 or 1 consecutive word tiles (1024 words each) of a query's bitmap,
# across segment boundaries: the most that still leaves 4 waves of 5 CTAs per SM. On 148 SMs:
# - 4096-doc segments (one 64-word tile each), 47 of them: 256 queries take 4, 128 take 2, 8 take 1;
# - 135168-doc segments (tiles of 1024, 1024 and 64 words), 16 of them, 256 queries: 4 tiles per CTA,
#   so CTAs start inside segments, and the last segment's last tiles lie past the last doc.
@pytest.mark.parametrize("seg_docs,n_docs,nq,check", [(4096, 190000, 256, 256), (4096, 190000, 128, 128),
                                                      (4096, 190000, 8, 8), (135168, 2030000, 256, 48)],
                         ids=["4_tiles", "2_tiles", "1_tile", "4_tiles_mid_segment"])
def test_batched_filter_tiles_across_segments(torch_cuda, seg_docs, n_docs, nq, check):
    torch = torch_cuda
    mix = data.Mixture(32, 64, (1e-3, 0.5), n_clusters=16, seed=91)
    vec, bits, _ = mix.corpus(n_docs, seed=92)
    table = hss.DataTable.build(vec, bits, 64, device=0, doc_num_per_segment=seg_docs)
    info = table.info
    exprs = data.make_filters(mix, nq, n_tags=(1, 6), seed=93)
    s = hss.FullRecallSearcher(table, max_batch=nq, candidate_cap=4096)
    f = s.compile_filters(exprs)
    words = info["segment_num"] * info["doc_num_per_segment"] // 64
    out = torch.zeros((nq, words), dtype=torch.int64, device="cuda")
    cnt = torch.zeros(nq, dtype=torch.int32, device="cuda")
    assert s.filter_device(f, nq, out.data_ptr(), words, cnt.data_ptr()) == _lib.HSS_OK
    got = out.cpu().numpy().view(np.uint64)
    counts = cnt.cpu().numpy()
    # every row, or rows spread over the batch (the oracle takes ~65 ms a filter at 2M docs)
    for i in np.linspace(0, nq - 1, check).astype(int):
        e = exprs[i]
        want = _bits_of(oracle.filter_bits(e, bits), n_docs)
        row = _bits_of(got[i], words * 64)
        assert (row[:n_docs] == want).all(), (i, e)
        assert not row[n_docs:].any(), (i, e)
        assert counts[i] == want.sum(), (i, e)


def test_filter_operator_both_table_conventions(torch_cuda):
    torch = torch_cuda
    mix, vec, bits, table = _table(torch, "bitmap", seed=5)
    info = table.info
    S, P = info["segment_num"], info["doc_num_per_segment"]
    rows_n = info["posting_rows"]
    _, ptab, _ = table.device_ptrs()
    # posting head addresses, row-major [rows][segments], read back through a torch copy
    nbytes = rows_n * S * 8
    heads = np.zeros(rows_n * S, np.uint64)
    tmp = torch.empty(rows_n * S, dtype=torch.int64, device="cuda")
    _copy_device(ptab, tmp.data_ptr(), nbytes)
    heads[:] = tmp.cpu().numpy().view(np.uint64)
    heads = heads.reshape(rows_n, S)
    words = S * P // 64
    for e in data.make_filters(mix, 25, n_tags=(1, 5), seed=21) + [x for x in _edge_filters() if x]:
        prog, rows, opn, empty = table.compile_filter(e)
        want = _bits_of(oracle.filter_bits(e, bits), vec.shape[0])
        for convention in ("heads", "reference"):
            tab = np.zeros((S, len(rows)), np.uint64)
            for si in range(S):
                for j, r in enumerate(rows):
                    a = int(heads[r, si])
                    if convention == "heads":
                        tab[si, j] = a
                        continue
                    # host copy of the same posting tells its layout and hit count
                    hdr = np.frombuffer(_host_head(table, r, si), np.uint32)
                    layout, hits = int(hdr[0]) >> 28, int(hdr[0]) & 0x0FFFFFFF
                    if r == rows_n - 1 or hits == 0:
                        tab[si, j] = 2  # EMPTY_OPERAND_TAG
                    elif layout == 0:
                        tab[si, j] = a + 8
                    else:
                        tab[si, j] = a | 1
            d_tab = torch.tensor(tab.reshape(-1).view(np.int64), device="cuda")
            d_prog = torch.tensor(prog.astype(np.int32), device="cuda")
            d_out = torch.zeros(words, dtype=torch.int64, device="cuda")
            d_status = torch.zeros(1, dtype=torch.int32, device="cuda")
            ctx = _lib.FilterContext(len(rows), S, P // 16, 1, len(prog), opn,
                                     _lib.HSS_FILTER_HEAD_ADDRESSES if convention == "heads" else 0)
            hss.bitmap_text_filter(d_tab.data_ptr(), d_prog.data_ptr(), ctx, d_out.data_ptr(), d_status.data_ptr())
            torch.cuda.synchronize()
            assert int(d_status.item()) == 0
            got = _bits_of(d_out.cpu().numpy().view(np.uint64), words * 64)[:vec.shape[0]]
            assert (got == want).all(), (e, convention)


def test_filter_operator_rejects_programs_whose_counts_would_wrap(torch_cuda):
    # Raw programs reach the operator as a device buffer, so the kernel's own program check is the
    # only guard. Operand and part counts near 2^32 would wrap a u32 sum (next + pn, pc + 2 + parts);
    # the check compares against the remaining room instead and reports the program as bad.
    torch = torch_cuda
    mix, vec, bits, table = _table(torch, "bitmap", seed=7)
    info = table.info
    S, P = info["segment_num"], info["doc_num_per_segment"]
    _, ptab, _ = table.device_ptrs()
    heads = torch.empty(info["posting_rows"] * S, dtype=torch.int64, device="cuda")
    _copy_device(ptab, heads.data_ptr(), heads.numel() * 8)
    _, rows, _, _ = table.compile_filter("5")
    tab = heads.view(info["posting_rows"], S)[int(rows[0])].contiguous()  # [segments], one operand
    big = 0xFFFFFFFF
    AND, OR, NOT, CONJ = 1, 2, 3, 0
    words = S * P // 64
    for prog in ([AND, 1, 0, AND, big, 1], [AND, 1, 0, CONJ, big], [NOT, big, 2], [OR, 1, 0, OR, big, 0],
                 [CONJ, 1, 1, AND, big, 1]):
        d_prog = torch.tensor(np.array(prog, np.uint32).view(np.int32), device="cuda")
        d_out = torch.full((words,), -1, dtype=torch.int64, device="cuda")
        d_status = torch.zeros(1, dtype=torch.int32, device="cuda")
        ctx = _lib.FilterContext(1, S, P // 16, 1, len(prog), 1, _lib.HSS_FILTER_HEAD_ADDRESSES)
        hss.bitmap_text_filter(tab.data_ptr(), d_prog.data_ptr(), ctx, d_out.data_ptr(), d_status.data_ptr())
        torch.cuda.synchronize()
        assert int(d_status.item()) & _lib.QSTATUS_BAD_PROGRAM, prog
        assert not d_out.cpu().numpy().any(), prog


_ROW_CACHE = {}


def _host_head(table, row, seg):
    toks = _ROW_CACHE.setdefault(id(table), _row_tokens(table))
    if row >= len(toks):
        return np.zeros(8, np.uint8).tobytes()
    b = table.posting(toks[row], seg)
    return b[:8] if b is not None else np.zeros(8, np.uint8).tobytes()


def _row_tokens(table):
    out = []
    for t in range(4096):
        tok = hss.hash64(str(t))
        if any(table.posting(tok, s) is not None for s in range(table.info["segment_num"])):
            out.append(tok)
        if len(out) == table.info["posting_rows"] - 1:
            break
    return out


def _copy_device(src_ptr, dst_ptr, nbytes):
    """Device-to-device copy between raw pointers (the library's table and a torch tensor)."""
    from cuda.bindings import runtime as rt
    err, = rt.cudaMemcpy(dst_ptr, src_ptr, nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
    assert int(err) == 0


@pytest.mark.parametrize("layout", ["bitmap", "packed", "matrix"])
def test_posting_bitlist_to_set_matches_oracle(torch_cuda, layout):
    torch = torch_cuda
    mix, vec, bits, table = _table(torch, layout, seed=7)
    info = table.info
    S, P = info["segment_num"], info["doc_num_per_segment"]
    rows_n = info["posting_rows"]
    _, ptab, _ = table.device_ptrs()
    tmp = torch.empty(rows_n * S, dtype=torch.int64, device="cuda")
    _copy_device(ptab, tmp.data_ptr(), rows_n * S * 8)
    heads = tmp.cpu().numpy().view(np.uint64).reshape(rows_n, S)
    srcs, want = [], []
    toks = _row_tokens(table)
    for r, tok in enumerate(toks):
        for si in range(S):
            b = table.posting(tok, si)
            if b is None:
                continue
            seg_docs = min(P, vec.shape[0] - si * P)
            srcs.append(int(heads[r, si]))
            full = np.zeros(P // 64, np.uint64)
            _, w = oracle.posting_decode(b, seg_docs)
            full[:w.size] = w
            want.append(full)
    out = torch.zeros((len(srcs), P // 64), dtype=torch.int64, device="cuda")
    dst = np.array([out.data_ptr() + i * (P // 8) for i in range(len(srcs))], np.uint64)
    d_src = torch.tensor(np.array(srcs, np.uint64).view(np.int64), device="cuda")
    d_dst = torch.tensor(dst.view(np.int64), device="cuda")
    hss.posting_bitlist_to_set(d_src.data_ptr(), P // 8, d_dst.data_ptr(), len(srcs))
    torch.cuda.synchronize()
    got = out.cpu().numpy().view(np.uint64)
    assert (got == np.stack(want)).all()


def _seq_scores(q, v):
    s = np.zeros(v.shape[0], np.float32)
    for d in range(v.shape[1]):
        s = (s + (v[:, d] * q[d]).astype(np.float32)).astype(np.float32)
    return s


@pytest.mark.parametrize("dim", [128, 36])
def test_vector_score_is_bit_exact(torch_cuda, dim):
    torch = torch_cuda
    rng = np.random.default_rng(dim)
    m, n = 37, 1000
    q = rng.standard_normal((m, dim)).astype(np.float32)
    v = rng.standard_normal((n, dim)).astype(np.float32)
    ld = n + 24
    dq, dv = torch.tensor(q, device="cuda"), torch.tensor(v, device="cuda")
    out = torch.zeros((m, ld), dtype=torch.float32, device="cuda")
    hss.vector_score(dq.data_ptr(), dv.data_ptr(), out.data_ptr(), m, n, dim, ld)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for i in range(m):
        assert (got[i, :n].view(np.uint32) == _seq_scores(q[i], v).view(np.uint32)).all()


@pytest.mark.parametrize("n", [1, 1000, 70001])
def test_aggregator_compacts_in_order(torch_cuda, n):
    torch = torch_cuda
    rng = np.random.default_rng(n)
    words = (n + 63) // 64 + 1
    bits = rng.integers(0, 2**63, words, dtype=np.int64).astype(np.uint64) & rng.integers(0, 2**63, words,
                                                                                            dtype=np.int64).astype(np.uint64)
    scores = rng.standard_normal(n).astype(np.float32)
    locs = rng.permutation(n).astype(np.uint32)
    keep = _bits_of(bits, n).astype(bool)
    d_bits = torch.tensor(bits.view(np.int64), device="cuda")
    d_sc = torch.tensor(scores, device="cuda")
    d_loc = torch.tensor(locs.view(np.int32), device="cuda")
    o_sc = torch.zeros(n, dtype=torch.float32, device="cuda")
    o_loc = torch.zeros(n, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    wsb = hss.aggregator_workspace_size(n)
    ws = torch.zeros(wsb, dtype=torch.uint8, device="cuda")
    hss.aggregator(d_bits.data_ptr(), d_sc.data_ptr(), d_loc.data_ptr(), o_sc.data_ptr(), o_loc.data_ptr(),
                   cnt.data_ptr(), n, ws.data_ptr(), wsb)
    torch.cuda.synchronize()
    c = int(cnt.item())
    assert c == keep.sum()
    assert (o_sc.cpu().numpy()[:c] == scores[keep]).all()
    assert (o_loc.cpu().numpy().view(np.uint32)[:c] == locs[keep]).all()


@pytest.mark.parametrize("n,k,levels", [(5000, 100, 0), (3000, 4096, 3), (100, 50, 0), (100, 200, 2),
                                        (200000, 1000, 7), (0, 10, 0)])
def test_topk_operator_is_exact_and_ordered(torch_cuda, n, k, levels):
    torch = torch_cuda
    rng = np.random.default_rng(n + k)
    scores = (rng.integers(0, levels, n).astype(np.float32) if levels else rng.standard_normal(n).astype(np.float32))
    locs = rng.permutation(max(n, 1))[:n].astype(np.uint32)
    # arrays of at least one element, so an empty list still passes non-null pointers
    d_sc = torch.tensor(np.concatenate([scores, np.zeros(1, np.float32)]), device="cuda")
    d_loc = torch.tensor(np.concatenate([locs, np.zeros(1, np.uint32)]).view(np.int32), device="cuda")
    d_n = torch.tensor([n], dtype=torch.int32, device="cuda")
    o_sc = torch.zeros(max(k, 1), dtype=torch.float32, device="cuda")
    o_loc = torch.zeros(max(k, 1), dtype=torch.int32, device="cuda")
    o_n = torch.zeros(1, dtype=torch.int32, device="cuda")
    hss.topk(d_sc.data_ptr(), d_loc.data_ptr(), d_n.data_ptr(), k, o_sc.data_ptr(), o_loc.data_ptr(), o_n.data_ptr())
    torch.cuda.synchronize()
    order = sorted(range(n), key=lambda i: (-scores[i], locs[i]))[:k]
    c = int(o_n.item())
    assert c == min(k, n)
    assert (o_loc.cpu().numpy().view(np.uint32)[:c] == locs[order]).all()
    assert (o_sc.cpu().numpy()[:c] == scores[order]).all()


def test_topk_operator_rejects_k_beyond_limit(torch_cuda):
    with pytest.raises(hss.HssError) as ei:
        hss.topk(1, 1, 1, _lib.HSS_MAX_TOPK + 1, 1, 1, 1)
    assert ei.value.code == _lib.HSS_ERR_LIMIT
