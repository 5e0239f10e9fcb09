"""Dense CPU oracle of weighted personalized PageRank and its gradient
(oracle/ppr_dense.py), checked without a GPU:

* T = 1 with unit weights reproduces the reference's PageRank (the golden
  PageRankHost outputs, hybrid_pr_host.cu:43-124, and the FP64 restatement
  sgso_pagerank);
* the closed-form adjoint gradient equals torch autograd through a dense
  solve, and both agree with central finite differences in FP64."""
import glob
import os

import numpy as np
import pytest

import oracle as O
import ppr_dense as D

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ALGO_FIX = sorted(glob.glob(os.path.join(GOLD, "ref_algos_*.npz")))


def _case(scale, seed, K, wseed=5):
    nv, row, col = O.rmat_csr(scale, 8, seed)
    rng = np.random.default_rng(wseed)
    w = np.exp(rng.uniform(np.log(0.1), np.log(10.0), len(col)))
    T = np.zeros((nv, K))
    for k in range(K):
        T[rng.choice(nv, 8, replace=False), k] = 1.0 / 8
    G = np.zeros((nv, K))
    G[rng.choice(nv, 16, replace=False)] = 1.0
    return nv, row, col, w, T, G


@pytest.mark.parametrize("path", ALGO_FIX, ids=os.path.basename)
def test_unit_ppr_is_reference_pagerank(path):
    f = np.load(path)
    nv, row, col = int(f["nv"]), f["row"], f["col"]
    X = D.ppr_dense(nv, row, col, np.ones(len(col)), np.ones((nv, 1)))[:, 0]
    assert np.max(np.abs(X - O.pagerank(nv, row, col))) < 1e-9
    ref = f["pr"].astype(np.float64)
    assert np.max(np.abs(ref - X) / X) < 1e-4


def test_parallel_edges_add_weight():
    # 0->1 twice (w 1, 2) and 0->2 (w 1): P[0,1] = 3/4
    row = np.array([0, 3, 3, 3], np.uint64)
    col = np.array([1, 1, 2], np.uint32)
    P, inv = D.dense_p(3, row, col, np.array([1.0, 2.0, 1.0]))
    assert P[0, 1] == pytest.approx(0.75) and P[0, 2] == pytest.approx(0.25)
    assert inv[1] == 0 and inv[2] == 0


@pytest.mark.parametrize("K", [1, 3])
def test_closed_gradient_equals_autograd(K):
    nv, row, col, w, T, G = _case(7, 2, K)
    X1, gw1, gT1 = D.ppr_grad_closed(nv, row, col, w, T, G)
    X2, gw2, gT2 = D.ppr_grad_autograd(nv, row, col, w, T, G)
    assert np.allclose(X1, X2, rtol=1e-12, atol=1e-14)
    assert np.allclose(gw1, gw2, rtol=1e-9, atol=1e-13)
    assert np.allclose(gT1, gT2, rtol=1e-9, atol=1e-13)


def test_closed_gradient_finite_differences():
    nv, row, col, w, T, G = _case(6, 4, 2)
    _, gw, gT = D.ppr_grad_closed(nv, row, col, w, T, G)
    rng = np.random.default_rng(9)
    L = lambda ww, TT: float((D.ppr_dense(nv, row, col, ww, TT) * G).sum())
    h = 1e-6
    d = rng.standard_normal(len(w)) * w
    fd = (L(w + h * d, T) - L(w - h * d, T)) / (2 * h)
    assert abs(fd - gw @ d) <= 1e-6 * max(abs(fd), 1e-12)
    dT = rng.standard_normal(T.shape)
    fd = (L(w, T + h * dT) - L(w, T - h * dT)) / (2 * h)
    assert abs(fd - (gT * dT).sum()) <= 1e-6 * max(abs(fd), 1e-12)


def test_sparse_jacobi_port_matches_dense():
    nv, row, col, w, T, _ = _case(8, 3, 3)
    X, k = D.ppr_jacobi_sparse(nv, row, col, w, T, tol=1e-14)
    assert k > 10
    assert np.allclose(X, D.ppr_dense(nv, row, col, w, T), rtol=1e-11, atol=1e-14)
