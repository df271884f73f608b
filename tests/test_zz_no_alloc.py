"""The allocation-free aggregator entry point (hss_aggregator_launch_noalloc), called through the
C-ABI and compared with the workspace entry point (hss_aggregator_launch) on the same inputs.

Two calls in a row share the library's one scratch array: the second call (a different, smaller
input) must not see anything the first left behind. The file is named to be collected last, so the
test also runs after every other GPU test in the same process; it passes alone as well."""

import numpy as np
import pytest

import hybridsearchsystem_b200 as hss
from hybridsearchsystem_b200 import _lib

pytestmark = pytest.mark.gpu


def _case(torch, n, seed):
    rng = np.random.default_rng(seed)
    words = (n + 63) // 64 + 1
    bits = rng.integers(0, 2**63, words, dtype=np.int64).astype(np.uint64) & \
        rng.integers(0, 2**63, words, dtype=np.int64).astype(np.uint64)
    scores = rng.standard_normal(n).astype(np.float32)
    locs = rng.permutation(n).astype(np.uint32)
    return (torch.tensor(bits.view(np.int64), device="cuda"), torch.tensor(scores, device="cuda"),
            torch.tensor(locs.view(np.int32), device="cuda"))


def _run(torch, fn, d_bits, d_sc, d_loc, n):
    o_sc = torch.full((n,), -7.0, dtype=torch.float32, device="cuda")
    o_loc = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    cnt = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    fn(o_sc, o_loc, cnt)
    torch.cuda.synchronize()
    c = int(cnt.item())
    return c, o_sc.cpu().numpy()[:c], o_loc.cpu().numpy().view(np.uint32)[:c]


def test_noalloc_aggregator_matches_workspace_entry_point(torch_cuda):
    torch = torch_cuda
    for n, seed in ((1_500_000, 1), (70_001, 2)):  # the second call is smaller than the first
        d_bits, d_sc, d_loc = _case(torch, n, seed)
        wsb = hss.aggregator_workspace_size(n)
        ws = torch.zeros(wsb, dtype=torch.uint8, device="cuda")
        want = _run(torch, lambda o, l, c: hss.aggregator(d_bits.data_ptr(), d_sc.data_ptr(), d_loc.data_ptr(),
                                                          o.data_ptr(), l.data_ptr(), c.data_ptr(), n,
                                                          ws.data_ptr(), wsb), d_bits, d_sc, d_loc, n)
        got = _run(torch, lambda o, l, c: hss.aggregator_noalloc(d_bits.data_ptr(), d_sc.data_ptr(),
                                                                 d_loc.data_ptr(), o.data_ptr(), l.data_ptr(),
                                                                 c.data_ptr(), n), d_bits, d_sc, d_loc, n)
        assert got[0] == want[0] > 0
        assert (got[1] == want[1]).all()
        assert (got[2] == want[2]).all()


def test_noalloc_aggregator_rejects_sizes_beyond_its_scratch(torch_cuda):
    torch = torch_cuda
    d = torch.zeros(4, dtype=torch.int64, device="cuda")
    lib = _lib.load()
    rc = lib.hss_aggregator_launch_noalloc(d.data_ptr(), d.data_ptr(), None, d.data_ptr(), d.data_ptr(),
                                           d.data_ptr(), _lib.HSS_AGGREGATOR_NOALLOC_MAX_DOCS + 1, None)
    assert rc == _lib.HSS_ERR_LIMIT
    assert b"HSS_AGGREGATOR_NOALLOC_MAX_DOCS" in lib.hss_last_error()
