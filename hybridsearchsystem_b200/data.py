"""Seeded synthetic inputs with the shapes and distributions of the benchmark configurations, and
the HYDSET2 file format they are exchanged in.

HYDSET2 (src/io/dataset_hw.h:1-98): a 40-byte header {magic "HYDSET2\\0", u32 version, u32 pad,
u64 doc_num, u32 vector_dim, u32 tag_num, u32 reserved, u32 pad}, then doc_num x dim float32, then
doc_num x ceil(tag_num/64) uint64 tag bitmaps (tag t = bit t%64 of word t/64).

Corpus: a mixture of Gaussian clusters (centres ~ N(0, I), point = centre + N(0, sigma^2 I)),
L2-normalised. Tags: tag t set independently with probability p_t, log-uniform over a range; a
number of tags are correlated with the cluster id (their probability is raised on a subset of
clusters and lowered elsewhere, keeping the marginal near p_t). Filters: random ASTs over a few
distinct tags joined by AND / OR / NOT, written in the reference's filter grammar.
"""
import math
import struct

import numpy as np

HYDSET2_HEADER = struct.Struct("<8sIIQIIII")


def write_hydset2(path, vectors, bits, tag_num):
    vectors = np.ascontiguousarray(vectors, np.float32)
    bits = np.ascontiguousarray(bits, np.uint64)
    n, dim = vectors.shape
    assert bits.shape == (n, (tag_num + 63) // 64)
    with open(path, "wb") as f:
        f.write(HYDSET2_HEADER.pack(b"HYDSET2\0", 2, 0, n, dim, tag_num, 0, 0))
        f.write(vectors.tobytes())
        f.write(bits.tobytes())


def read_hydset2(path):
    """Returns (vectors [n, dim] float32, bits [n, words] uint64, tag_num), memory-mapped."""
    with open(path, "rb") as f:
        magic, _ver, _p0, n, dim, tag_num, _r, _p1 = HYDSET2_HEADER.unpack(f.read(HYDSET2_HEADER.size))
    if magic[:7] != b"HYDSET2":
        raise ValueError("bad HYDSET2 magic")
    words = (tag_num + 63) // 64
    mm = np.memmap(path, dtype=np.uint8, mode="r")
    off = HYDSET2_HEADER.size
    vec = mm[off:off + n * dim * 4].view(np.float32).reshape(n, dim)
    off += n * dim * 4
    bits = mm[off:off + n * words * 8].view(np.uint64).reshape(n, words)
    return vec, bits, tag_num


class Mixture:
    """Cluster mixture and tag model shared by the corpus and its queries."""

    def __init__(self, dim, tag_num, p_range, n_clusters=1024, sigma=0.3, n_corr=16, corr_frac=1.0 / 16,
                 corr_boost=8.0, seed=1):
        rng = np.random.default_rng(seed)
        self.dim, self.tag_num, self.sigma = dim, tag_num, sigma
        self.n_clusters = n_clusters
        self.centres = rng.standard_normal((n_clusters, dim)).astype(np.float32)
        lo, hi = p_range
        self.p = np.exp(rng.uniform(math.log(lo), math.log(hi), tag_num))
        n_corr = min(n_corr, tag_num)
        self.corr_tags = rng.choice(tag_num, n_corr, replace=False)
        k = max(1, int(round(corr_frac * n_clusters)))
        self.corr_clusters = [rng.choice(n_clusters, k, replace=False) for _ in range(n_corr)]
        self.corr_boost = corr_boost
        self.corr_frac = k / n_clusters
        self.seed = seed

    def tag_prob(self, t, cluster_ids):
        """Per-doc probability of tag t."""
        p = self.p[t]
        j = np.nonzero(self.corr_tags == t)[0]
        if j.size == 0:
            return np.full(cluster_ids.shape, p, np.float64)
        hi = min(1.0, p * self.corr_boost)
        lo = max(0.0, (p - self.corr_frac * hi) / (1.0 - self.corr_frac))
        inside = np.isin(cluster_ids, self.corr_clusters[j[0]])
        return np.where(inside, hi, lo)

    def _points(self, rng, n):
        cid = rng.integers(0, self.n_clusters, n)
        x = self.centres[cid] + self.sigma * rng.standard_normal((n, self.dim)).astype(np.float32)
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        return x.astype(np.float32), cid

    def corpus(self, n, seed=None, chunk=1 << 20):
        """(vectors [n, dim] float32, tag bits [n, ceil(tag_num/64)] uint64, cluster ids)."""
        rng = np.random.default_rng(self.seed * 1000003 + 17 if seed is None else seed)
        words = (self.tag_num + 63) // 64
        vec = np.empty((n, self.dim), np.float32)
        bits = np.zeros((n, words), np.uint64)
        cids = np.empty(n, np.int64)
        for a in range(0, n, chunk):
            b = min(n, a + chunk)
            v, cid = self._points(rng, b - a)
            vec[a:b] = v
            cids[a:b] = cid
            for t in range(self.tag_num):
                hit = rng.random(b - a) < self.tag_prob(t, cid)
                bits[a:b, t // 64] |= hit.astype(np.uint64) << np.uint64(t % 64)
        return vec, bits, cids

    def corpus_torch(self, n, device="cuda", seed=None, chunk=1 << 21):
        """The same model drawn with torch on a GPU (fast for 10M-doc corpora; a different stream of
        random numbers than corpus()). Returns host numpy arrays (vectors, tag bits)."""
        vec = np.empty((n, self.dim), np.float32)

        def sink(a, b, x):
            vec[a:b] = x.float().cpu().numpy()

        bits = self._draw_torch(n, device, seed, chunk, sink)
        return vec, bits

    def corpus_device(self, n, device="cuda", seed=None, chunk=1 << 20):
        """As corpus_torch, but the vectors stay on the device: (torch tensor [n, dim] float32 on
        `device`, host tag bits). For corpora larger than host memory should hold twice."""
        import torch
        vec = torch.empty((n, self.dim), dtype=torch.float32, device=device)

        def sink(a, b, x):
            vec[a:b] = x

        bits = self._draw_torch(n, device, seed, chunk, sink)
        return vec, bits

    def _draw_torch(self, n, device, seed, chunk, sink):
        import torch
        g = torch.Generator(device=device)
        g.manual_seed(self.seed * 1000003 + 29 if seed is None else seed)
        words = (self.tag_num + 63) // 64
        centres = torch.tensor(self.centres, device=device)
        bits = np.zeros((n, words), np.uint64)
        p = torch.tensor(self.p, device=device, dtype=torch.float32)
        corr_mask = torch.zeros(self.tag_num, self.n_clusters, dtype=torch.bool, device=device)
        for j, t in enumerate(self.corr_tags):
            corr_mask[int(t), torch.tensor(self.corr_clusters[j], device=device)] = True
        is_corr = torch.zeros(self.tag_num, dtype=torch.bool, device=device)
        is_corr[torch.tensor(self.corr_tags, device=device)] = True
        hi = torch.clamp(p * self.corr_boost, max=1.0)
        lo = torch.clamp((p - self.corr_frac * hi) / (1.0 - self.corr_frac), min=0.0)
        shifts = torch.arange(64, device=device, dtype=torch.int64)
        for a in range(0, n, chunk):
            b = min(n, a + chunk)
            m = b - a
            cid = torch.randint(0, self.n_clusters, (m,), generator=g, device=device)
            x = centres[cid] + self.sigma * torch.randn((m, self.dim), generator=g, device=device)
            x = x / torch.linalg.norm(x, dim=1, keepdim=True)
            sink(a, b, x)
            del x
            u = torch.rand((m, self.tag_num), generator=g, device=device)
            prob = p.expand(m, -1)
            inside = corr_mask[:, cid].T  # [m, tag_num]
            prob = torch.where(is_corr & inside, hi.expand(m, -1), torch.where(is_corr, lo.expand(m, -1), prob))
            hit = (u < prob).to(torch.int64)
            pad = words * 64 - self.tag_num
            if pad:
                hit = torch.nn.functional.pad(hit, (0, pad))
            w = (hit.view(m, words, 64) << shifts).sum(dim=2)  # bits are disjoint: sum == or
            bits[a:b] = w.cpu().numpy().view(np.uint64)
        return bits

    def queries(self, nq, seed=2):
        rng = np.random.default_rng(seed)
        v, _ = self._points(rng, nq)
        return v

    def selectivity(self, ast):
        """Estimated pass fraction of an AST under tag independence."""
        op = ast[0]
        if op == "T":
            return float(self.p[ast[1]])
        if op == "N":
            return 1.0 - self.selectivity(ast[1])
        vals = [self.selectivity(c) for c in ast[1]]
        if op == "A":
            return float(np.prod(vals))
        return 1.0 - float(np.prod([1.0 - v for v in vals]))


def ast_text(ast, top=True):
    """The reference grammar's text of an AST ("T", tag) / ("N", child) / ("A"|"O", [children])."""
    op = ast[0]
    if op == "T":
        return str(int(ast[1]))
    if op == "N":
        return "NOT " + ast_text(ast[1], False)
    s = (" AND " if op == "A" else " OR ").join(ast_text(c, False) for c in ast[1])
    return s if top else "(" + s + ")"


def random_ast(rng, tag_num, n_tags, p_not=0.2, p_and=0.6):
    tags = rng.choice(tag_num, n_tags, replace=False)
    items = [("N", ("T", int(t))) if rng.random() < p_not else ("T", int(t)) for t in tags]
    while len(items) > 1:
        i = int(rng.integers(0, len(items) - 1))
        op = "A" if rng.random() < p_and else "O"
        a, b = items[i], items[i + 1]
        kids = (a[1] if a[0] == op else [a]) + (b[1] if b[0] == op else [b])
        items[i:i + 2] = [(op, kids)]
    return items[0]


def make_filters(mix, nq, n_tags=(1, 4), seed=3, selectivity_range=None, pool_factor=24):
    """nq filter texts. With selectivity_range=(lo, hi), ASTs are picked so that their estimated
    selectivities spread log-uniformly over the range."""
    rng = np.random.default_rng(seed)

    def draw():
        return random_ast(rng, mix.tag_num, int(rng.integers(n_tags[0], n_tags[1] + 1)))

    if selectivity_range is None:
        return [ast_text(draw()) for _ in range(nq)]
    lo, hi = (math.log(x) for x in selectivity_range)
    pool = [draw() for _ in range(nq * pool_factor)]
    logsel = np.array([math.log(max(1e-12, mix.selectivity(a))) for a in pool])
    targets = rng.uniform(lo, hi, nq)
    return [ast_text(pool[j]) for j in _nearest_unused(logsel, targets)]


def _nearest_unused(values, targets):
    """For each target in turn, the index of the unused value nearest to it (lowest index among equally
    near ones), which is then used: the greedy match, in O((n + m) log n) with a sorted order and
    skip pointers over used positions."""
    n = len(values)
    order = np.lexsort((np.arange(n), values))  # by value, then index
    sv = values[order]
    # start of each run of equal values in sorted order (its lowest index comes first)
    run_start = np.zeros(n, np.int64)
    for i in range(1, n):
        run_start[i] = run_start[i - 1] if sv[i] == sv[i - 1] else i
    right = list(range(n + 1))  # right[i]: first unused position >= i (n: none)
    left = list(range(-1, n))   # left[i + 1]: last unused position <= i (-1: none)

    def find(ptr, i, off):
        root = i
        while ptr[root + off] != root:
            root = ptr[root + off]
        while ptr[i + off] != root:  # path compression
            ptr[i + off], i = root, ptr[i + off]
        return root

    out = []
    for t in targets:
        pos = int(np.searchsorted(sv, t))
        best = None
        r = find(right, pos, 0) if pos < n else n
        if r < n:
            best = (abs(sv[r] - t), order[r], r)
        lpos = find(left, pos - 1, 1) if pos > 0 else -1
        if lpos >= 0:
            # the lowest unused index among the values equal to the left neighbour
            l = find(right, int(run_start[lpos]), 0)
            c = (abs(sv[l] - t), order[l], l)
            if best is None or (c[0], c[1]) < (best[0], best[1]):
                best = c
        _, j, p = best
        right[p] = p + 1
        left[p + 1] = p - 1
        out.append(int(j))
    return out


# Benchmark configurations (corpus shapes and distributions).
CONFIGS = {
    # plain exact method, one segment: 131,072 docs x 128, 64 tags, batch 32, top-100
    "cfg1": dict(n=131072, dim=128, tag_num=64, p_range=(1e-3, 0.5), n_tags=(1, 4), nq=1000, batch=32,
                 topk=(100,), selectivity_range=None, doc_num_per_segment=131072),
    # plain exact method at scale: 10M x 128, 256 tags, K in {10, 100, 1000}, batches 64 / 256
    "cfg2": dict(n=10_000_000, dim=128, tag_num=256, p_range=(1e-4, 0.6), n_tags=(1, 6), nq=10000, batch=256,
                 topk=(10, 100, 1000), selectivity_range=(1e-4, 1.0), doc_num_per_segment=131072),
}
