"""sgs_sssp_csr_noalloc: the entry point for callers that cannot allocate
device memory (code inside an allocator hook or a memory-pool callback, where
an allocation would re-enter the allocator; embedders with memory fixed at
start-up).  It must give the same distances and parents as the engine's
regular SSSP/BFS queries, on two calls in a row (its scratch is a static
device array reused by every call), and reject every input its checks cover
with the documented status, leaving the next correct call exact.

Collected last on purpose (file name) so that a run stopping at the first
failure has run everything else first."""
import ctypes

import numpy as np
import pytest

import oracle as O
import sgs

pytestmark = pytest.mark.gpu


def _fn():
    L = sgs.lib()
    f = L.sgs_sssp_csr_noalloc
    f.argtypes = [ctypes.c_uint32] + [ctypes.c_void_p] * 3 + [ctypes.c_uint32] + [ctypes.c_void_p] * 3
    f.restype = ctypes.c_int
    return f


def test_noalloc_matches_engine_queries():
    import torch

    fn = _fn()
    nv, row, col = O.rmat_csr(16, 16, 3)
    w = O.weights(nv, row, col, 7, 0)
    with sgs.Engine() as e:
        e.load_csr(nv, row, col, w)
        qs, qb = e.add_query(sgs.SSSP, 0), e.add_query(sgs.BFS, 11)
        ref = {"sssp": (qs.value(), qs.parent()), "bfs": (qb.value(), qb.parent())}
    # values must equal the engine's; parents (not unique) must be valid tight
    # predecessors, and this kernel keeps the smallest-id one, like the oracle
    exact = {"sssp": O.sssp(nv, row, col, w, 0)[1], "bfs": O.bfs(nv, row, col, 11)[1]}
    weights = {"sssp": w, "bfs": None}
    dev = torch.device("cuda", 0)
    d_row = torch.from_numpy(row.view(np.int64)).to(dev)
    d_col = torch.from_numpy(col.view(np.int32)).to(dev)
    d_w = torch.from_numpy(w.view(np.int32)).to(dev)
    dist = torch.empty(nv, dtype=torch.int32, device=dev)
    par = torch.empty(nv, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    for name, wp, src in (("sssp", d_w.data_ptr(), 0), ("bfs", None, 11)):
        for call in range(2):  # the static scratch keeps the previous call's contents
            dist.fill_(-7)
            par.fill_(-7)
            torch.cuda.synchronize()
            rc = fn(nv, d_row.data_ptr(), d_col.data_ptr(), wp, src, dist.data_ptr(),
                    par.data_ptr(), None)
            torch.cuda.synchronize()
            assert rc == 0, sgs.lib().sgs_last_error()
            got_d = dist.cpu().numpy().view(np.uint32)
            got_p = par.cpu().numpy().view(np.uint32)
            assert np.array_equal(got_d, ref[name][0]), (name, call)
            assert np.array_equal(got_p, exact[name]), (name, call)
            assert O.check_tree(nv, row, col, weights[name], src, got_d, ref[name][1]) == 0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    fn = _fn()
    dev = torch.device("cuda", 0)
    d_row = torch.zeros(4, dtype=torch.int64, device=dev)
    d_col = torch.zeros(1, dtype=torch.int32, device=dev)
    dist = torch.empty(4, dtype=torch.int32, device=dev)
    rc = fn((1 << 20) + 1, d_row.data_ptr(), d_col.data_ptr(), None, 0, dist.data_ptr(), None, None)
    assert rc == -1
    assert b"nv must be" in sgs.lib().sgs_last_error()


def _dev_csr(row, col, w=None):
    import torch

    dev = torch.device("cuda", 0)
    t = [torch.from_numpy(np.ascontiguousarray(row, np.uint64).view(np.int64)).to(dev),
         torch.from_numpy(np.ascontiguousarray(col, np.uint32).view(np.int32)).to(dev)]
    t.append(None if w is None else
             torch.from_numpy(np.ascontiguousarray(w, np.uint32).view(np.int32)).to(dev))
    return t


def _call(fn, nv, row, col, w, src):
    import torch

    d_row, d_col, d_w = _dev_csr(row, col, w)
    dist = torch.empty(max(nv, 1), dtype=torch.int32, device=d_row.device)
    par = torch.empty(max(nv, 1), dtype=torch.int32, device=d_row.device)
    torch.cuda.synchronize()
    rc = fn(nv, d_row.data_ptr(), d_col.data_ptr(), None if d_w is None else d_w.data_ptr(), src,
            dist.data_ptr(), par.data_ptr(), None)
    torch.cuda.synchronize()
    return rc, dist.cpu().numpy().view(np.uint32)[:nv], par.cpu().numpy().view(np.uint32)[:nv]


def test_noalloc_rejects_bad_csr_and_recovers():
    """Every documented rejection returns its status and message without
    touching memory outside the caller's arrays, and a correct call right
    after it is exact again.  Each bad input is one the entry point checks
    before use: the offsets on the host (row[0], row[nv] against the edge
    limit) or in its first kernel (decreasing rows, before any edge is read),
    destinations and weights per edge before they index anything."""
    fn = _fn()
    nv, row, col = O.rmat_csr(10, 8, 4)
    w = O.weights(nv, row, col, 5, 0)
    good_d = O.sssp(nv, row, col, w, 0)[0]
    u32 = lambda x: np.array(x, np.uint32)  # noqa: E731
    u64 = lambda x: np.array(x, np.uint64)  # noqa: E731
    cases = [
        # (nv, row, col, w, status, message part)
        (4, u64([1, 2, 3, 4, 5]), u32([1, 2, 3, 0, 1]), None, -1, b"start at 0"),
        (4, u64([0, 3, 1, 4, 4]), u32([1, 2, 3, 0]), None, -1, b"not decrease"),
        (4, u64([0, 1, 2, 3, 3]), u32([1, 99, 3]), None, -1, b"destination"),
        (4, u64([0, 1, 2, 3, 3]), u32([1, 2, 3]), u32([5, 0, 5]), -1, b"weight 0"),
        (4, u64([0, 0, 0, 0, (1 << 25) + 1]), u32([0]), None, -1, b"edges"),
    ]
    for k, (n, r, c, ww, status, msg) in enumerate(cases):
        rc, _, _ = _call(fn, n, r, c, ww, 0)
        assert rc == status, (k, rc)
        assert msg in sgs.lib().sgs_last_error(), (k, sgs.lib().sgs_last_error())
        rc, d, p = _call(fn, nv, row, col, w, 0)
        assert rc == 0, (k, sgs.lib().sgs_last_error())
        assert np.array_equal(d, good_d), k
        assert O.check_tree(nv, row, col, w, 0, d, p) == 0, k


def test_noalloc_round_limit_then_exact():
    """A path longer than the round limit (1000 rounds) ends with
    SGS_ERR_NOCONV; the next call is exact again."""
    fn = _fn()
    n = 1100
    row = np.arange(n + 1, dtype=np.uint64)
    row[-1] = n - 1  # vertex n-1 has no out-edge
    col = np.arange(1, n, dtype=np.uint32)
    rc, _, _ = _call(fn, n, row, col, None, 0)
    assert rc == -5
    assert b"round limit" in sgs.lib().sgs_last_error()
    nv, row2, col2 = O.rmat_csr(10, 8, 6)
    rc, d, p = _call(fn, nv, row2, col2, None, 3)
    assert rc == 0
    assert np.array_equal(d, O.bfs(nv, row2, col2, 3)[0])
    assert O.check_tree(nv, row2, col2, None, 3, d, p) == 0
