"""Differentiable weighted personalized PageRank on the GPU (sgs_ppr_* through
the C ABI and sgs.autograd), against the dense CPU oracle:

* forward: T = 1 with unit weights equals the reference's PageRank (FP64
  restatement pinned to PageRankHost); weighted K-vector forward equals the
  dense solve for K = 1, 3, 8, 33, 64, 100 (every lane layout of the kernels)
  and on hub vertices whose edges are split into pieces;
* backward: per-edge and teleport gradients equal torch autograd through a
  dense CPU solve, and central finite differences of the GPU forward in FP64
  on a scale-12 R-MAT graph (directional and single-edge, rel 1e-4);
* torch.autograd.Function: loss.backward() gives the same gradients, float32
  inputs get float32 gradients, gradcheck on a small graph;
* errors: bad weights, bad CSR, bad alpha or K raise, the handle stays usable.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
import ppr_dense as D
import sgs

pytestmark = pytest.mark.gpu

ALPHA = 0.85


def _graph(scale, seed=1, ef=16):
    return O.rmat_csr(scale, ef, seed)


def _weights(ne, seed=5):
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(0.1), np.log(10.0), ne))


def _teleport(nv, K, seeds=32, seed=7):
    rng = np.random.default_rng(seed)
    T = np.zeros((nv, K))
    for k in range(K):
        T[rng.choice(nv, seeds, replace=False), k] = 1.0 / seeds
    return T


def _targets(nv, n=256, K=1, seed=11):
    rng = np.random.default_rng(seed)
    G = np.zeros((nv, K))
    G[rng.choice(nv, n, replace=False)] = 1.0
    return G


def test_unit_weights_all_ones_is_pagerank():
    nv, row, col = _graph(12, 3)
    with sgs.Ppr(nv, row, col) as g:
        X = g.forward(np.ones(g.ne), np.ones((nv, 1)))[:, 0]
    assert np.max(np.abs(X - O.pagerank(nv, row, col))) < 1e-9


@pytest.mark.parametrize("K", [1, 3, 8, 33, 64, 100])
def test_forward_matches_dense(K):
    nv, row, col = _graph(11, 2)
    w = _weights(len(col), K)
    T = _teleport(nv, K, 16, K)
    with sgs.Ppr(nv, row, col) as g:
        r2, c2 = g.export()
        assert np.array_equal(r2, row) and np.array_equal(c2, col)
        X = g.forward(w, T)
        assert g.last_iters > 10
    ref = D.ppr_dense(nv, row, col, w, T)
    assert np.max(np.abs(X - ref)) <= 1e-10 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("K", [1, 5, 40])
def test_hub_vertices_split_into_pieces(K):
    """Vertex 0 has 3000 out-edges and vertex 1 3000 in-edges (several
    pieces each, one of them partial) besides a random background graph."""
    rng = np.random.default_rng(K)
    nv = 3100
    src = np.concatenate([np.zeros(3000), rng.integers(2, nv, 3000), rng.integers(0, nv, 6000)])
    dst = np.concatenate([rng.integers(0, nv, 3000), np.ones(3000), rng.integers(0, nv, 6000)])
    row, col = O.csr_from_edges(nv, src.astype(np.uint32), dst.astype(np.uint32), dedupe=False)
    w = _weights(len(col), 3)
    T = _teleport(nv, K, 20, 4)
    G = _targets(nv, 64, K, 9)
    G[1] = 1.0
    tol = 1e-16 * nv * K
    with sgs.Ppr(nv, row, col) as g:
        X = g.forward(w, T, tol=tol)
        gw, gT = g.backward(w, X, G, tol=tol)
    Xr, gw_r, gT_r = D.ppr_grad_closed(nv, row, col, w, T, G)
    assert np.max(np.abs(X - Xr)) <= 1e-10 * np.abs(Xr).max()
    assert np.max(np.abs(gw - gw_r)) <= 1e-9 * np.abs(gw_r).max()
    assert np.max(np.abs(gT - gT_r)) <= 1e-9 * np.abs(gT_r).max()


@pytest.mark.parametrize("K", [1, 4, 33])
def test_backward_matches_dense_autograd(K):
    nv, row, col = _graph(11, 4)
    w = _weights(len(col), 3)
    T = _teleport(nv, K, 16, 1)
    G = _targets(nv, 128, K)
    with sgs.Ppr(nv, row, col) as g:
        X = g.forward(w, T)
        gw, gT = g.backward(w, X, G)
    _, gw_ref, gT_ref = D.ppr_grad_autograd(nv, row, col, w, T, G)
    scale_w = np.abs(gw_ref).max()
    assert np.max(np.abs(gw - gw_ref)) <= 1e-9 * scale_w
    assert np.max(np.abs(gT - gT_ref)) <= 1e-9 * np.abs(gT_ref).max()
    _, gw_c, _ = D.ppr_grad_closed(nv, row, col, w, T, G)
    assert np.max(np.abs(gw - gw_c)) <= 1e-9 * scale_w


def test_finite_differences_scale12_fp64():
    """Central differences of the GPU forward itself (FP64, scale 12),
    relative error 1e-4: random directions in w and T, and single edges."""
    nv, row, col = _graph(12, 1)
    K = 4
    w = _weights(len(col), 2)
    T = _teleport(nv, K, 32, 3)
    G = _targets(nv, 256, K, 5)
    rng = np.random.default_rng(0)
    with sgs.Ppr(nv, row, col) as g:
        tol = 1e-15 * nv * K
        X = g.forward(w, T, tol=tol)
        gw, gT = g.backward(w, X, G, tol=tol)
        L = lambda ww, TT: float((g.forward(ww, TT, tol=tol) * G).sum())
        h = 1e-5
        for _ in range(3):
            d = rng.standard_normal(len(w)) * w
            fd = (L(w + h * d, T) - L(w - h * d, T)) / (2 * h)
            an = float(gw @ d)
            assert abs(fd - an) <= 1e-4 * abs(fd), (fd, an)
            dT = rng.standard_normal(T.shape) * (T > 0)
            fd = (L(w, T + h * dT) - L(w, T - h * dT)) / (2 * h)
            an = float((gT * dT).sum())
            assert abs(fd - an) <= 1e-4 * abs(fd), (fd, an)
        # the largest single-edge gradients, one edge at a time
        for e in np.argsort(-np.abs(gw))[:8]:
            he = 1e-4 * w[e]
            wp, wm = w.copy(), w.copy()
            wp[e] += he
            wm[e] -= he
            fd = (L(wp, T) - L(wm, T)) / (2 * he)
            assert abs(fd - gw[e]) <= 1e-4 * abs(fd), (e, fd, gw[e])


def test_autograd_function_float32_inputs():
    import torch

    from sgs.autograd import personalized_pagerank

    nv, row, col = _graph(10, 6)
    K = 2
    w = _weights(len(col), 8)
    T = _teleport(nv, K, 8, 2)
    G = _targets(nv, 64, K, 3)
    with sgs.Ppr(nv, row, col) as g:
        wt = torch.tensor(w, dtype=torch.float32, device="cuda", requires_grad=True)
        Tt = torch.tensor(T, dtype=torch.float32, device="cuda", requires_grad=True)
        X = personalized_pagerank(g, wt, Tt)
        assert X.dtype == torch.float64 and X.shape == (nv, K)
        loss = (X * torch.tensor(G, device="cuda")).sum()
        loss.backward()
        assert wt.grad.dtype == torch.float32 and Tt.grad.dtype == torch.float32
        _, gw_ref, gT_ref = D.ppr_grad_autograd(nv, row, col, w.astype(np.float32).astype(np.float64),
                                                T.astype(np.float32).astype(np.float64), G)
    gw = wt.grad.double().cpu().numpy()
    assert np.max(np.abs(gw - gw_ref)) <= 1e-6 * np.abs(gw_ref).max()
    assert np.max(np.abs(Tt.grad.double().cpu().numpy() - gT_ref)) <= 1e-6 * np.abs(gT_ref).max()


def test_autograd_gradcheck_small():
    import torch

    from sgs.autograd import personalized_pagerank

    rng = np.random.default_rng(1)
    nv = 12
    src = rng.integers(0, nv, 40)
    dst = rng.integers(0, nv, 40)
    row, col = O.csr_from_edges(nv, src.astype(np.uint32), dst.astype(np.uint32), dedupe=False)
    with sgs.Ppr(nv, row, col) as g:
        wt = torch.tensor(_weights(len(col), 4), device="cuda", requires_grad=True)
        Tt = torch.tensor(rng.random((nv, 3)), device="cuda", requires_grad=True)
        f = lambda a, b: personalized_pagerank(g, a, b, tol=1e-15 * nv * 3)
        assert torch.autograd.gradcheck(f, (wt, Tt), eps=1e-6, atol=1e-7, rtol=1e-5)


def test_prepared_from_engine_snapshot():
    """sgs_ppr_create on an engine: the current (updated) graph, whose unit
    PPR equals both the oracle PageRank and the engine's own PR query."""
    nv, row, col = _graph(11, 9)
    w = O.weights(nv, row, col, 1, 0)
    with sgs.Engine() as e:
        e.load_csr(nv, row, col, w)
        q = e.add_query(sgs.PR, 0)
        i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 3, 500, 500)
        iw = np.array([O.weight_of(1, u, v) for u, v in zip(i_s, i_d)], np.uint32)
        e.apply_batch(i_s, i_d, iw, d_s, d_d)
        row2, col2, _ = O.apply(nv, row, col, w, i_s, i_d, iw, d_s, d_d)
        with sgs.Ppr(engine=e) as g:
            r, c = g.export()
            assert np.array_equal(r, row2)
            for v in range(0, nv, 97):
                assert sorted(c[r[v]:r[v + 1]]) == sorted(col2[row2[v]:row2[v + 1]])
            X = g.forward(np.ones(g.ne), np.ones((nv, 1)))[:, 0]
        assert np.max(np.abs(X - O.pagerank(nv, row2, col2))) < 1e-9
        assert np.max(np.abs(X - q.value())) < 1e-5


def test_edge_cases_and_errors():
    # no edges: X = (1 - alpha) T, gradients of T only
    row = np.zeros(6, np.uint64)
    col = np.zeros(0, np.uint32)
    with sgs.Ppr(5, row, col) as g:
        T = np.arange(10, dtype=np.float64).reshape(5, 2)
        X = g.forward(np.zeros(0), T)
        assert np.allclose(X, (1 - ALPHA) * T)
        gw, gT = g.backward(np.zeros(0), X, np.ones((5, 2)))
        assert len(gw) == 0 and np.allclose(gT, (1 - ALPHA))
    nv, row, col = _graph(8, 1)
    with sgs.Ppr(nv, row, col) as g:
        w = _weights(g.ne)
        T = np.ones((nv, 1))
        for bad in (0.0, -1.0, np.nan, np.inf):
            wb = w.copy()
            wb[17] = bad
            with pytest.raises(sgs.SgsError):
                g.forward(wb, T)
        for a in (0.0, 1.0, 1.5):
            with pytest.raises(sgs.SgsError):
                g.forward(w, T, alpha=a)
        with pytest.raises(sgs.SgsError):  # step limit
            g.forward(w, T, max_iter=3)
        L = sgs.lib()
        X = np.empty((nv, 1))
        it = ctypes.c_int()
        assert L.sgs_ppr_forward(g.h, w.ctypes.data, T.ctypes.data, 0, ALPHA, 1e-9, 100,
                                 X.ctypes.data, ctypes.byref(it), sgs.MEM_HOST) == -1
        # still usable after the errors
        X = g.forward(w, T)
        assert np.allclose(X, D.ppr_dense(nv, row, col, w, T), rtol=1e-9, atol=1e-12)
    bad_col = col.copy()
    bad_col[3] = nv
    with pytest.raises(sgs.SgsError):
        sgs.Ppr(nv, row, bad_col)
    bad_row = row.copy()
    bad_row[5] = bad_row[6] + 1
    with pytest.raises(sgs.SgsError):
        sgs.Ppr(nv, bad_row, col)
