"""sgs_sssp_csr_noalloc: the entry point for callers that cannot allocate
device memory (allocator hooks, code running during someone else's graph
capture, embedders with memory fixed at start-up).  It must give the same
distances and parents as the engine's regular SSSP/BFS queries, on two calls
in a row (its scratch is a static device array reused by every call).

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
