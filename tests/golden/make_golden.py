"""Generates the golden fixtures in this directory from the reference's OWN code.

Run in a checkout where the reference sources were compiled (`make -C oracle` builds
oracle/_ref/libref.so from them). The fixtures pin the oracle (oracle.c) and the product's host codec to
the reference:
  hash64.npz     Hash64 (hash.cpp) of decimal tag tokens and random strings
  postings.npz   PostingSerializer::Serialize output for id sets x layouts (SPARSE_PACKED cases are
                 produced in a child process with NPUR_SPARSE_PACKED=1, which the serializer reads once)
  filters.json   ParseFilter accept/reject and EvalFilterBitmap results over probe bitmaps
  topk.npz       CpuTopK (fp32 mode) id sets on small corpora, tie-heavy ones included, and
                 CpuTopKBatch sets on the same inputs

Usage: python tests/golden/make_golden.py
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
os.environ.setdefault("NPUR_LOG_LEVEL", "ERROR")

import oracle  # noqa: E402


def posting_cases(rng):
    cases = []
    for seg_docs in (16, 17, 100, 1000, 4096, 131072):
        for density in (0.0, 0.001, 0.01, 1 / 64, 0.05, 0.3, 1.0):
            n = int(round(density * seg_docs))
            ids = np.sort(rng.choice(seg_docs, n, replace=False)).astype(np.uint32) if n else np.zeros(0, np.uint32)
            for is_matrix in (0, 1):
                for thr in (1 / 64, 0.05, -1.0):
                    cases.append((ids, seg_docs, is_matrix, thr))
    return cases


def serialize_all(cases):
    r = oracle.ref()
    out = []
    for ids, seg_docs, is_matrix, thr in cases:
        cap = 8 + max(seg_docs, 6 * ((seg_docs + 15) // 16), 4 * ids.size) + 64
        buf = np.zeros(cap, np.uint8)
        n = r.ref_posting_serialize(ids.ctypes.data, ids.size, seg_docs, is_matrix, thr, buf.ctypes.data, cap)
        assert n >= 0
        out.append(buf[:n].copy())
    return out


def main_packed_child(path_in, path_out):
    d = np.load(path_in, allow_pickle=True)
    cases = list(d["cases"])
    blobs = serialize_all(cases)
    np.save(path_out, np.array(blobs, dtype=object), allow_pickle=True)


def make_hash():
    r = oracle.ref()
    rng = np.random.default_rng(11)
    tokens = [str(i) for i in range(4096)] + ["".join(chr(int(c)) for c in rng.integers(32, 127, int(n)))
                                              for n in rng.integers(0, 48, 256)]
    hashes = np.array([r.ref_hash64(t.encode(), len(t.encode())) for t in tokens], np.uint64)
    np.savez_compressed(os.path.join(HERE, "hash64.npz"), tokens=np.array(tokens, dtype=object), hashes=hashes)


def make_postings():
    rng = np.random.default_rng(12)
    cases = posting_cases(rng)
    blobs = serialize_all(cases)
    tmp_in = os.path.join(HERE, "_cases.npy.npz")
    tmp_out = os.path.join(HERE, "_packed.npy")
    np.savez(tmp_in, cases=np.array(cases, dtype=object))
    env = dict(os.environ, NPUR_SPARSE_PACKED="1")
    subprocess.check_call([sys.executable, __file__, "--packed-child", tmp_in, tmp_out], env=env)
    packed = list(np.load(tmp_out, allow_pickle=True))
    os.remove(tmp_in)
    os.remove(tmp_out)
    np.savez_compressed(os.path.join(HERE, "postings.npz"),
                        ids=np.array([c[0] for c in cases], dtype=object),
                        seg_docs=np.array([c[1] for c in cases], np.uint32),
                        is_matrix=np.array([c[2] for c in cases], np.int32),
                        threshold=np.array([c[3] for c in cases], np.float32),
                        plain=np.array(blobs, dtype=object), packed=np.array(packed, dtype=object))


def make_filters():
    r = oracle.ref()
    exprs = [
        "47", "47 AND 48", "47 OR 48", "NOT 47", "1 OR 2 AND 3", "NOT 1 AND 2", "(1 OR 2) AND 3",
        "(1 OR 2) AND NOT (3 OR 4)", "NOT NOT 5", "NOT (1 AND 2)", "1 AND 2 AND 3 AND 4", "1 OR 2 OR 3 OR 4",
        "", "   ", "\t\n", "(1 OR 2", "1 OR 2)", "()", "AND 2", "1 AND", "1 2", "1 OR OR 2", "NOT",
        "0", "63", "64", "0 AND 63 AND 64", "127 OR 128", "255", "256", "1000", "35839",
        "1 and 2", "1 AND2", "NOT5", "1AND 2", "((((3))))", "(3) AND ((4 OR 5) AND NOT (6))", "1 & 2",
        "18446744073709551615", "18446744073709551616", "00012", " 7 ", "NOTX 5", "( 1 OR ( 2 AND 3 ) )",
        "((47 AND (12 OR 31 OR 30) AND (46 OR 11)) AND (NOT (25 OR 15)) AND 9)",
    ]
    rng = np.random.default_rng(13)
    sys.path.insert(0, ROOT)
    from hybridsearchsystem_b200 import data
    mix = data.Mixture(16, 192, (0.01, 0.6), n_clusters=8, seed=5)
    exprs += data.make_filters(mix, 120, n_tags=(1, 6), seed=14)
    words = 4
    probes = rng.integers(0, 2**63, (64, words), dtype=np.int64).astype(np.uint64)
    probes[0] = 0
    probes[1] = np.uint64(0xFFFFFFFFFFFFFFFF)
    probes[2] = [1, 0, 0, 0]
    probes[3] = [1 << 63, 1, 0, 0]
    sparse = rng.random((60, words * 64)) < 0.15
    for i in range(60):
        w = np.zeros(words, np.uint64)
        for t in np.nonzero(sparse[i])[0]:
            w[t // 64] |= np.uint64(1) << np.uint64(t % 64)
        probes[4 + i] = w
    result = []
    for e in exprs:
        ok = r.ref_parse_ok(e.encode())
        ev = [r.ref_eval_bitmap(e.encode(), p.ctypes.data, words) for p in probes] if ok else []
        result.append({"expr": e, "ok": int(ok), "eval": ev})
    with open(os.path.join(HERE, "filters.json"), "w") as f:
        json.dump({"words": words, "probes": [[int(x) for x in p] for p in probes], "cases": result}, f)


def make_topk():
    r = oracle.ref()
    rng = np.random.default_rng(15)
    sys.path.insert(0, ROOT)
    from hybridsearchsystem_b200 import data
    corpora = []
    # (name, docs, dim, tags, value levels (0 = continuous), nq, topk)
    specs = [("random", 1500, 16, 128, 0, 24, 40), ("levels8", 1500, 16, 128, 8, 24, 40),
             ("levels3", 1500, 16, 128, 3, 24, 40), ("levels2", 1500, 16, 128, 2, 24, 40),
             ("k_over_hits", 300, 16, 128, 0, 16, 5000), ("more_queries_than_docs", 120, 16, 128, 4, 150, 20)]
    out = {}
    for name, n, dim, tags, levels, nq, k in specs:
        if levels:
            vec = rng.integers(0, levels, (n, dim)).astype(np.float32)
            q = rng.integers(0, levels, (nq, dim)).astype(np.float32)
        else:
            vec = (np.round(rng.uniform(-1, 1, (n, dim)) * 256) / 256).astype(np.float32)
            q = (np.round(rng.uniform(-1, 1, (nq, dim)) * 256) / 256).astype(np.float32)
        words = (tags + 63) // 64
        bits = np.zeros((n, words), np.uint64)
        hit = rng.random((n, tags)) < 0.2
        for t in range(tags):
            bits[:, t // 64] |= hit[:, t].astype(np.uint64) << np.uint64(t % 64)
        mix = data.Mixture(dim, tags, (0.05, 0.5), n_clusters=4, seed=16)
        exprs = data.make_filters(mix, nq, n_tags=(1, 3), seed=17)
        for i in range(0, nq, 7):
            exprs[i] = ""  # match all
        topks = np.array([k if i % 3 == 0 else k // 2 + 1 for i in range(nq)], np.int32)
        cap = int(topks.max())
        single = np.full((nq, cap), -1, np.int64)
        scount = np.zeros(nq, np.int32)
        for i in range(nq):
            buf = np.zeros(cap, np.int64)
            c = r.ref_cpu_topk(q[i].ctypes.data, dim, exprs[i].encode(), vec.ctypes.data, bits.ctypes.data, tags, n, 0,
                               int(topks[i]), 1, buf.ctypes.data, cap)
            assert c >= 0
            single[i, :c] = buf[:c]
            scount[i] = c
        import ctypes
        arr = (ctypes.c_char_p * nq)(*[e.encode() for e in exprs])
        batch = np.full((nq, cap), -1, np.int64)
        bcount = np.zeros(nq, np.int32)
        rc = r.ref_cpu_topk_batch(q.ctypes.data, nq, dim, arr, topks.ctypes.data, vec.ctypes.data, bits.ctypes.data,
                                  tags, n, 0, 1, 2, cap, batch.ctypes.data, bcount.ctypes.data)
        assert rc == 0
        for key, val in (("vectors", vec), ("bits", bits), ("queries", q), ("topks", topks),
                         ("single_ids", single), ("single_counts", scount), ("batch_ids", batch),
                         ("batch_counts", bcount), ("tag_num", np.int32(tags))):
            out[f"{name}__{key}"] = val
        out[f"{name}__filters"] = np.array(exprs, dtype=object)
        corpora.append(name)
    out["corpora"] = np.array(corpora, dtype=object)
    np.savez_compressed(os.path.join(HERE, "topk.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--packed-child":
        main_packed_child(sys.argv[2], sys.argv[3])
        sys.exit(0)
    if not oracle.ref_available():
        sys.exit("oracle/_ref/libref.so not built: run `make -C oracle` where the reference sources exist")
    make_hash()
    make_postings()
    make_filters()
    make_topk()
    print("golden fixtures written to", HERE)
