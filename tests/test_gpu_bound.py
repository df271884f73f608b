"""The proven error bound of the tensor-core candidate pass under adversarial rows, through the C-ABI.

Every tensor-core form is exact only if its approximate score s~ stays within the query's bound
E_q of the ground truth's FP32 score s (sequential over d, multiply then add) for every doc, since
the thresholds are lowered by E_q. Two corpora drive the bound where it is tightest:

1. Truncation: rows exactly representable in TF32, BF16 and E4M3 with per-vector scale (so the
   quantisation terms of E_q vanish and only the accumulation model remains). Coordinate 0 of every
   query and doc dominates (1.75 * 1.75); the other products are all positive and sit a chosen
   number of bits below it, the range where aligning the addends to the largest and cutting them to
   p bits loses the most. Each group of docs targets a different offset, so whatever the hardware's
   accumulation width, some group straddles it.
2. Cancellation: FP32 rows that are not representable and not normalised: alternating-sign
   coordinates of large magnitude, per-coordinate magnitudes spread over 2^-20..1 and per-row norms
   over 1e-3..1e3, so sums cancel heavily and the quantisation terms are large.

Each case asserts |s~ - s| <= E_q over every doc (all docs are candidates: K >= corpus size) on the
one-SM pass (40 queries) and the SM-pair pass (200 queries), checks the final results bit-exact
against the oracle, and prints the largest |s~ - s| / E_q. The truncation case also prints the
accumulation error against an exact (FP64) sum as a fraction of the model's bound, and the
effective accumulation width in bits that fraction implies."""
import numpy as np
import pytest

import hybridsearchsystem_b200 as hss
import oracle

pytestmark = pytest.mark.gpu

METHODS = {"tf32": 1, "bf16": 2, "e4m3": 3}
# instruction K (terms per MMA) and the bits the accumulation model assumes (one below the measured)
MODEL = {"tf32": (8, 23), "bf16": (16, 23), "e4m3": (32, 13)}
N_DOCS = 2048


def _seq_scores(q, v):
    """The ground truth's FP32 score of every (query, doc): sequential over d, each product and sum
    rounded to FP32 (no contraction)."""
    s = np.zeros((q.shape[0], v.shape[0]), np.float32)
    for d in range(v.shape[1]):
        s = (s + (q[:, d:d + 1] * v[None, :, d]).astype(np.float32)).astype(np.float32)
    return s


def _e4m3_values(rng, exps, n):
    """Positive values (1 + m/8) 2^e with e from `exps` (exactly representable in E4M3, BF16, TF32)."""
    m = rng.integers(0, 8, n)
    return ((1.0 + m / 8.0) * np.exp2(exps)).astype(np.float32)


def _truncation_rows(rng, n, dim, q_exps=None, target=None):
    """Rows with coordinate 0 = 1.75 (= 448 * 2^-8, so the E4M3 per-vector scale is 2^-8 exactly) and
    coordinates 1.. positive with exponents in [-14, -1] (E4M3 normals at that scale)."""
    x = np.zeros((n, dim), np.float32)
    x[:, 0] = 1.75
    for r in range(n):
        if q_exps is None:
            e = rng.integers(-14, 0, dim - 1)
        else:
            # product exponent e_q + e_v aimed at target[r], within the representable range
            e = np.clip(target[r] - q_exps[1:], -14, -1)
        x[r, 1:] = _e4m3_values(rng, e, dim - 1)
    return x


def _cancellation_rows(rng, n, dim):
    mag = np.exp2(rng.uniform(-20.0, 0.0, (n, dim)))
    sign = np.where(np.arange(dim) % 2 == 0, 1.0, -1.0)[None, :] * np.where(rng.random((n, 1)) < 0.5, 1.0, -1.0)
    x = mag * sign * (1.0 + 0.01 * rng.standard_normal((n, dim)))
    scale = np.exp(rng.uniform(np.log(1e-3), np.log(1e3), (n, 1)))
    return (x / np.linalg.norm(x, axis=1, keepdims=True) * scale).astype(np.float32)


def _run(method, vec, q, what):
    n, dim = vec.shape
    nq = q.shape[0]
    bits = np.full((n, 1), np.uint64(0xFFFFFFFFFFFFFFFF), np.uint64)
    table = hss.DataTable.build(vec, bits, 64, device=0, doc_num_per_segment=1024)
    s = hss.FullRecallSearcher(table, max_batch=256, method=METHODS[method])
    k = hss._lib.HSS_MAX_TOPK  # above the corpus size: the threshold stays -inf, every doc is a candidate
    for a in q:
        s.add_query("", a, k)
    scores, ids, counts = s.batch_search()
    seq = _seq_scores(q, vec)
    worst = 0.0
    approx = np.zeros((nq, n), np.float64)
    for i in range(nq):
        sc, loc, cnt, theta, eps = s.last_candidates(i)
        assert cnt == n and len(loc) == n, (what, method, i, cnt)
        assert np.isneginf(theta)
        approx[i, loc] = sc
        dev = np.abs(sc.astype(np.float64) - seq[i, loc].astype(np.float64))
        worst = max(worst, float(dev.max() / eps))
        assert (dev <= eps).all(), (what, method, i, float(dev.max()), eps)
    ws, wi, wc = oracle.topk(q, [""] * nq, k, vec, bits, threads=8)
    for i in range(nq):
        c = int(wc[i])
        assert int(counts[i]) == c == n
        assert (ids[i][:c] == wi[i][:c]).all(), (what, method, i)
        assert (scores[i][:c].view(np.uint32) == ws[i][:c].view(np.uint32)).all(), (what, method, i)
    s.close()
    table.close()
    return worst, approx


@pytest.mark.parametrize("dim", [128, 768])
@pytest.mark.parametrize("nq", [40, 200], ids=["one_sm", "sm_pair"])
@pytest.mark.parametrize("method", list(METHODS))
def test_accumulation_bound_under_truncation(torch_cuda, method, nq, dim):
    rng = np.random.default_rng(1000 + dim + nq)
    q = _truncation_rows(rng, nq, dim)
    # every query shares coordinate 0; doc exponents aim the products at offsets of 10..28 bits below
    # the dominant product, in groups of docs (query 0's exponents set the aim; the others scatter)
    targets = np.repeat(np.arange(-27, -9, 2), N_DOCS // 9 + 1)[:N_DOCS]
    q_exps = np.floor(np.log2(q[0])).astype(np.int64)
    vec = _truncation_rows(rng, N_DOCS, dim, q_exps=q_exps, target=targets)
    worst, approx = _run(method, vec, q, "truncation")
    # accumulation error against the exact sum (products of these values are exact in FP64 and their
    # sum spans fewer than 53 bits), as a fraction of the model's bound
    exact = q.astype(np.float64) @ vec.astype(np.float64).T
    nrm = np.linalg.norm(q.astype(np.float64), axis=1)[:, None] * np.linalg.norm(vec.astype(np.float64), axis=1)[None, :]
    kk, p = MODEL[method]
    steps = -(-dim // kk)
    model = (dim + 2 * steps) * 2.0 ** (1 - p)
    rel = np.abs(approx - exact) / nrm
    frac = float(rel.max() / model)
    bits_eff = float(1 - np.log2(max(rel.max(), 1e-300) / (dim + 2 * steps)))
    at = int(targets[np.argmax(rel.max(axis=0))])
    print(f"\n[bound] truncation {method} dim={dim} nq={nq}: max |s~-s|/E_q = {worst:.4f}; accumulation error "
          f"{rel.max():.3e} of |q||v| = {frac:.4f} of the model (p={p}); effective width >= {bits_eff:.1f} bits "
          f"(worst doc group aimed 2^{at} below the dominant product)")
    assert frac <= 1.0


@pytest.mark.parametrize("nq", [40, 200], ids=["one_sm", "sm_pair"])
@pytest.mark.parametrize("method", list(METHODS))
def test_bound_under_cancellation(torch_cuda, method, nq):
    rng = np.random.default_rng(2000 + nq)
    vec = _cancellation_rows(rng, N_DOCS, 128)
    q = _cancellation_rows(rng, nq, 128)
    worst, _ = _run(method, vec, q, "cancellation")
    print(f"\n[bound] cancellation {method} nq={nq}: max |s~-s|/E_q = {worst:.4f}")
