"""The product's host library on the CPU: libhss.so loads and exports every symbol include/hss.h
declares; its Hash64, posting writer, filter grammar and filter-program compiler agree with the
golden vectors and the oracle; the index directory round-trips through the reference's posting-file
format. No GPU is touched (tables are built host-only, device = -1)."""
import json
import os
import re
import struct

import numpy as np
import pytest

import hybridsearchsystem_b200 as hss
import oracle
from hybridsearchsystem_b200 import _lib, data

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    with open(os.path.join(ROOT, "include", "hss.h")) as f:
        header = f.read()
    declared = set(re.findall(r"\b(hss_\w+)\s*\(", header))
    lib = _lib.load()
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert declared == bound, declared ^ bound


def test_hash64_matches_reference(golden):
    g = golden("hash64.npz")
    got = np.array([hss.hash64(t) for t in g["tokens"]], np.uint64)
    assert (got == g["hashes"]).all()


@pytest.mark.parametrize("packed", [False, True])
def test_posting_writer_matches_reference(golden, packed):
    g = golden("postings.npz")
    for i in range(len(g["seg_docs"])):
        want = bytes(g["packed" if packed else "plain"][i])
        got = hss.posting_serialize(g["ids"][i], int(g["seg_docs"][i]), bool(g["is_matrix"][i]),
                                    float(g["threshold"][i]), packed)
        if (want[3] >> 4) == 3:
            assert got[:8] == want[:8]
            assert sorted(np.frombuffer(got[8:], np.uint32)) == sorted(np.frombuffer(want[8:], np.uint32))
        else:
            assert got == want, i


def _small_table(seed=0, n=5000, tags=96, p=1024, **kw):
    mix = data.Mixture(32, tags, (0.002, 0.6), n_clusters=16, seed=seed)
    vec, bits, _ = mix.corpus(n, seed=seed + 100)
    return mix, vec, bits, hss.DataTable.build(vec, bits, tags, device=-1, doc_num_per_segment=p, **kw)


def test_filter_grammar_matches_reference(golden):
    _, _, _, table = _small_table()
    g = golden("filters.json")
    for case in g["cases"]:
        try:
            table.compile_filter(case["expr"])
            ok = True
        except hss.HssError as e:
            assert e.code == _lib.HSS_ERR_PARSE
            ok = False
        assert ok == bool(case["ok"]), case["expr"]


def _check_programs(mix, vec, bits, table, exprs, p):
    info = table.info
    segs = info["segment_num"]
    n = vec.shape[0]
    for e in exprs:
        prog, rows, opn, empty = table.compile_filter(e)
        want = oracle.filter_bits(e, bits)
        if empty:
            assert oracle.Parsed(e).root < 0
            continue
        got = np.zeros(segs * p // 64, np.uint64)
        for s in range(segs):
            seg_docs = min(p, n - s * p)
            operands = []
            for r in rows:
                tok = None if r == info["posting_rows"] - 1 else r
                blob = None if tok is None else _posting_of_row(table, r, s)
                if blob is None:
                    operands.append(np.zeros(p // 64, np.uint64))
                else:
                    layout, w = oracle.posting_decode(blob, seg_docs)
                    assert layout >= 0
                    full = np.zeros(p // 64, np.uint64)
                    full[:w.size] = w
                    operands.append(full)
            out = oracle.eval_postfix(prog, opn, operands, p // 64)
            assert out is not None, e
            got[s * p // 64:(s + 1) * p // 64] = out
        got_bits = np.unpackbits(got.view(np.uint8), bitorder="little")[:n]
        want_bits = np.unpackbits(want.view(np.uint8), bitorder="little")[:n]
        assert (got_bits == want_bits).all(), e


_ROW_TOKENS = {}


def _posting_of_row(table, row, seg):
    # rows are assigned to the tags present in the corpus in ascending tag order
    tokens = _ROW_TOKENS.setdefault(id(table), _row_tokens(table))
    return table.posting(tokens[row], seg)


def _row_tokens(table):
    out = []
    for t in range(4096):
        tok = hss.hash64(str(t))
        if any(table.posting(tok, s) is not None for s in range(table.info["segment_num"])):
            out.append(tok)
        if len(out) == table.info["posting_rows"] - 1:
            break
    return out


@pytest.mark.parametrize("layout", ["bitmap", "packed", "matrix"])
def test_compiled_programs_equal_ground_truth_filter(layout):
    kw = {"bitmap": {}, "packed": {"sparse_packed": True}, "matrix": {"matrix_posting": True}}[layout]
    mix, vec, bits, table = _small_table(seed=3, **kw)
    exprs = data.make_filters(mix, 40, n_tags=(1, 6), seed=9)
    exprs += ["", "5", "NOT 5", "NOT NOT 7", "1 AND 1", "200 OR 3", "NOT 250", "3 AND NOT 3", "(1 OR 2) AND (3 OR 4)"]
    _check_programs(mix, vec, bits, table, exprs, 1024)


def test_index_layouts_cover_all_five_codes():
    seen = set()
    for kw in ({}, {"sparse_packed": True}, {"matrix_posting": True}):
        _, _, _, table = _small_table(seed=4, **kw)
        for t in range(96):
            for s in range(table.info["segment_num"]):
                b = table.posting(hss.hash64(str(t)), s)
                if b is not None:
                    seen.add(b[3] >> 4)
    assert seen == {0, 1, 2, 3, 4}


def test_index_directory_roundtrip_in_reference_posting_format(tmp_path):
    mix, vec, bits, table = _small_table(seed=5)
    table.save(tmp_path)
    segs = table.info["segment_num"]
    # the posting files follow the reference's layout (inverted_builder.cpp:178-250)
    for s in range(segs):
        path = tmp_path / "content" / f"poissonengine_1_{s}_content.posting"
        raw = path.read_bytes()
        ver, = struct.unpack_from("<B", raw, 0)
        ext_len, = struct.unpack_from("<H", raw, 6)
        assert ver == 1 and ext_len == 1 and raw[8:9] == b"1"
        token_num, = struct.unpack_from("<I", raw, 9)
        for i in range(token_num):
            tok, po, to = struct.unpack_from("<QII", raw, 13 + 16 * i)
            lit_len, = struct.unpack_from("<I", raw, to)
            lit = raw[to + 4:to + 4 + lit_len].decode()
            assert hss.hash64(lit) == tok
            assert raw[po:po + 8] == table.posting(tok, s)[:8]
    loaded = hss.DataTable.load(tmp_path, device=-1)
    assert loaded.info == table.info
    for t in range(0, 96, 5):
        tok = hss.hash64(str(t))
        for s in range(segs):
            assert loaded.posting(tok, s) == table.posting(tok, s)
    exprs = data.make_filters(mix, 10, n_tags=(1, 4), seed=12)
    for e in exprs:
        a, b = table.compile_filter(e), loaded.compile_filter(e)
        assert (a[0] == b[0]).all() and (a[1] == b[1]).all()


def test_corrupt_posting_file_is_rejected(tmp_path):
    _, _, _, table = _small_table(seed=6, n=2048)
    table.save(tmp_path)
    path = tmp_path / "content" / "poissonengine_1_0_content.posting"
    raw = bytearray(path.read_bytes())
    token_num, = struct.unpack_from("<I", raw, 9)
    _, po, _ = struct.unpack_from("<QII", raw, 13)
    raw[po + 3] = (raw[po + 3] & 0x0F) | 0x70  # layout code 7: unknown
    path.write_bytes(bytes(raw))
    with pytest.raises(hss.HssError) as ei:
        hss.DataTable.load(tmp_path, device=-1)
    assert ei.value.code == _lib.HSS_ERR_INDEX


def test_index_config_is_validated():
    vec = np.zeros((10, 8), np.float32)
    bits = np.zeros((10, 1), np.uint64)
    with pytest.raises(hss.HssError):
        hss.DataTable.build(vec, bits, 8, device=-1, doc_num_per_segment=100)  # not a multiple of 128
    with pytest.raises(hss.HssError):
        hss.DataTable.build(np.zeros((10, 6), np.float32), bits, 8, device=-1, doc_num_per_segment=128)  # dim % 4


def _ref_half(x):
    """The reference's own Float32ToFloat16 (trans_number.cpp:38-83) of every float in x."""
    r = oracle.ref()
    return np.array([r.ref_f32_to_f16(float(v)) for v in np.ravel(x)], np.uint16).reshape(np.shape(x))


@pytest.mark.skipif(not oracle.ref_available(), reason="needs the reference's CPU build (oracle/_ref)")
def test_reference_index_directory_roundtrip(tmp_path):
    # write the reference's own index layout (fr_builder's output: meta, id mapping, FP16 Zn vector
    # blocks, posting files) and read it back the way its DataTable::LoadData does
    mix, vec, bits, table = _small_table(seed=7, n=3000, tags=96, p=1024)
    vec = vec.copy()
    # edge values of the FP16 conversion: halfway cases, values that flush to zero, overflow
    vec[0, :8] = [1.0 + 2.0 ** -11, 1.0 + 3 * 2.0 ** -11, 2.0 ** -15, -2.0 ** -25, 65504.0, 65520.0, -70000.0, 0.0]
    table = hss.DataTable.build(vec, bits, 96, device=-1, doc_num_per_segment=1024)
    zn = 16
    table.save_reference(tmp_path, zn)
    segs, dim, n = table.info["segment_num"], vec.shape[1], vec.shape[0]
    meta = json.loads((tmp_path / "poissonengine_1.meta").read_text())
    assert meta == {"config": {"docNumPerSegment": 1024, "splitDocNumZn": zn},
                    "schema": {"posting": ["content"], "vector": ["content"]},
                    "statistics": {"docNum": n, "segmentNum": segs}}
    want_half = _ref_half(vec)
    groups = (dim + 15) // 16
    for s in range(segs):
        d0, seg_docs = s * 1024, min(1024, n - s * 1024)
        idm = (tmp_path / "id" / f"poissonengine_1_{s}.idm").read_bytes()
        assert idm[:9] == bytes([1, 0, 0, 0, 0, 0, 1, 0]) + b"0"
        assert (np.frombuffer(idm[9:], np.uint64) == np.arange(d0, d0 + seg_docs)).all()
        raw = (tmp_path / "content" / f"poissonengine_1_{s}_content.vector").read_bytes()
        assert raw[:8] == bytes([1, 0, 0, 0, 0, 0, 2, 0]) and struct.unpack_from("<H", raw, 8)[0] == dim
        body = np.frombuffer(raw[10:], np.uint16)
        assert body.size == -(-seg_docs // zn) * zn * groups * 16  # the last segment padded to whole blocks
        # doc l, dims 16j..16j+15 sit at (l // zn) * zn * groups * 16 + (zn * j + l % zn) * 16
        # (vector_builder.cpp:52-56)
        for l in (0, 1, zn - 1, zn, seg_docs - 1):
            for j in range(groups):
                at = (l // zn) * zn * groups * 16 + (zn * j + l % zn) * 16
                assert (body[at:at + 16] == want_half[d0 + l, 16 * j:16 * j + 16]).all(), (s, l, j)
    loaded = hss.DataTable.load_reference(tmp_path, device=-1)
    assert loaded.info["doc_num"] == n and loaded.info["segment_num"] == segs and loaded.info["dim"] == dim
    for t in range(0, 96, 3):
        tok = hss.hash64(str(t))
        for s in range(segs):
            assert loaded.posting(tok, s) == table.posting(tok, s)
    for e in data.make_filters(mix, 20, n_tags=(1, 4), seed=13):
        a, b = table.compile_filter(e), loaded.compile_filter(e)
        assert (a[0] == b[0]).all() and (a[1] == b[1]).all()
    # the loaded rows are the FP16 values, widened exactly
    loaded.save(tmp_path / "own")
    got = np.fromfile(tmp_path / "own" / "vectors.f32", np.float32).reshape(n, dim)
    r = oracle.ref()
    want = np.array([r.ref_f16_to_f32(int(h)) for h in want_half.ravel()], np.float32).reshape(n, dim)
    assert (got.view(np.uint32) == want.view(np.uint32)).all() or \
        np.array_equal(np.isnan(got), np.isnan(want)) and (got[~np.isnan(got)] == want[~np.isnan(want)]).all()
    assert loaded.load_times["vector_bytes"] == n * dim * 4


def test_reference_index_directory_rejections(tmp_path):
    mix, vec, bits, table = _small_table(seed=8, n=600, tags=16, p=256)
    table.save_reference(tmp_path, 16)
    meta = tmp_path / "poissonengine_1.meta"
    text = meta.read_text()
    meta.write_text(text.replace('"docNumPerSegment":256', '"docNumPerSegment":200'))
    with pytest.raises(hss.HssError):
        hss.DataTable.load_reference(tmp_path, device=-1)  # not a multiple of 128
    meta.write_text(text)
    idm = tmp_path / "id" / "poissonengine_1_0.idm"
    raw = bytearray(idm.read_bytes())
    raw[8:9] = b"1"  # string doc ids
    idm.write_bytes(bytes(raw))
    with pytest.raises(hss.HssError):
        hss.DataTable.load_reference(tmp_path, device=-1)


def test_searcher_workspace_bytes_follow_the_configuration():
    _, _, _, table = _small_table(seed=11, n=4000, tags=32, p=1024)
    ws = hss.FullRecallSearcher.workspace_bytes
    small = ws(table, max_batch=16, candidate_cap=1 << 14)
    assert small > 16 * (1 << 14) * 16  # candidate lists (score + location) and the select workspace
    assert ws(table, max_batch=32, candidate_cap=1 << 14) > small
    assert ws(table, max_batch=16, candidate_cap=1 << 15) > small
    # the tensor-core methods add the staged query tile; the candidate cap never drops below 4096
    assert ws(table, max_batch=16, candidate_cap=1 << 14, method=2) > small
    assert ws(table, max_batch=16, candidate_cap=1) == ws(table, max_batch=16, candidate_cap=4096)
