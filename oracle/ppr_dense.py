"""Dense CPU oracle for weighted personalized PageRank and its gradient
(TEST INFRASTRUCTURE ONLY: imported by ``tests/`` as the checker).

The fixed point generalises the reference's PageRank
(samples/hybrid_pr/hybrid_pr.cu:26-151; host form PageRankHost in
samples/hybrid_pr/hybrid_pr_host.cu:43): with P[u, v] = w_uv / s_u, s_u = sum
of u's out-edge weights (parallel edges add up; rows without out-edges stay
zero, so their mass is dropped as in the reference),

    X = (1 - alpha) T + alpha P^T X        (one column per teleport vector)

T = 1 with unit weights gives the reference's unnormalised PageRank, which
``sgs_oracle.c:sgso_pagerank`` restates by power iteration.

Two gradients are offered for a loss L with dL/dX = G:

* :func:`ppr_grad_closed` -- the adjoint formulas (Y = G + alpha P Y,
  dL/dT = (1 - alpha) Y, dL/dw_uv = sum_k X[u,k] (alpha Y[v,k] - Y[u,k] +
  G[u,k]) / s_u) evaluated with dense solves;
* :func:`ppr_grad_autograd` -- torch autograd through a dense CPU solve of
  the same fixed point, built from the edge weights, which shares no formula
  with the adjoint above.

Dense: nv up to a few thousand.
"""
from __future__ import annotations

import numpy as np


def _src(nv, row):
    return np.repeat(np.arange(nv, dtype=np.int64), np.diff(row.astype(np.int64)))


def dense_p(nv, row, col, w):
    """Row-normalised dense transition matrix P (float64) and 1/s."""
    src = _src(nv, row)
    dst = col.astype(np.int64)
    w = np.asarray(w, np.float64)
    s = np.zeros(nv)
    np.add.at(s, src, w)
    inv = np.where(s > 0, 1.0 / np.where(s > 0, s, 1.0), 0.0)
    P = np.zeros((nv, nv))
    np.add.at(P, (src, dst), w * inv[src])
    return P, inv


def ppr_dense(nv, row, col, w, T, alpha=0.85):
    """X solving (I - alpha P^T) X = (1 - alpha) T; T is [nv, K]."""
    P, _ = dense_p(nv, row, col, w)
    A = np.eye(nv) - alpha * P.T
    return np.linalg.solve(A, (1.0 - alpha) * np.asarray(T, np.float64).reshape(nv, -1))


def ppr_grad_closed(nv, row, col, w, T, G, alpha=0.85):
    """(X, dL/dw per edge, dL/dT) from the adjoint formulas, dense solves."""
    P, inv = dense_p(nv, row, col, w)
    T = np.asarray(T, np.float64).reshape(nv, -1)
    G = np.asarray(G, np.float64).reshape(nv, -1)
    X = np.linalg.solve(np.eye(nv) - alpha * P.T, (1.0 - alpha) * T)
    Y = np.linalg.solve(np.eye(nv) - alpha * P, G)
    src = _src(nv, row)
    dst = col.astype(np.int64)
    term = (X[src] * (alpha * Y[dst] - Y[src] + G[src])).sum(axis=1)
    return X, term * inv[src], (1.0 - alpha) * Y


def ppr_grad_autograd(nv, row, col, w, T, G, alpha=0.85):
    """(X, dL/dw, dL/dT) by torch autograd through a dense CPU solve, L = <G, X>."""
    import torch

    src = torch.from_numpy(_src(nv, row))
    dst = torch.from_numpy(col.astype(np.int64))
    wt = torch.tensor(np.asarray(w, np.float64), requires_grad=True)
    Tt = torch.tensor(np.asarray(T, np.float64).reshape(nv, -1), requires_grad=True)
    s = torch.zeros(nv, dtype=torch.float64).index_add(0, src, wt)
    p = wt / s[src]
    PT = torch.zeros(nv, nv, dtype=torch.float64).index_put((dst, src), p, accumulate=True)
    A = torch.eye(nv, dtype=torch.float64) - alpha * PT
    X = torch.linalg.solve(A, (1.0 - alpha) * Tt)
    L = (X * torch.from_numpy(np.asarray(G, np.float64).reshape(nv, -1))).sum()
    L.backward()
    return X.detach().numpy(), wt.grad.numpy(), Tt.grad.numpy()


def sparse_pt(nv, row, col, w):
    """P^T as a scipy CSR matrix."""
    import scipy.sparse as sp

    w = np.asarray(w, np.float64)
    src = _src(nv, row)
    s = np.bincount(src, weights=w, minlength=nv)
    inv = np.where(s > 0, 1.0 / np.where(s > 0, s, 1.0), 0.0)
    return sp.csr_matrix((w * inv[src], (col.astype(np.int64), src)), shape=(nv, nv))


def ppr_jacobi_sparse(nv, row, col, w, T, alpha=0.85, iters=None, tol=None, X0=None, PT=None):
    """The same Jacobi iteration the GPU runs, X <- (1 - alpha) T + alpha P^T X,
    on the CPU with a scipy CSR matrix (single thread): for the timed CPU
    baseline.  Runs `iters` steps, or until the L1 step change is below tol.
    Returns (X, steps)."""
    if PT is None:
        PT = sparse_pt(nv, row, col, w)
    T = np.asarray(T, np.float64).reshape(nv, -1)
    B = (1.0 - alpha) * T
    X = B.copy() if X0 is None else X0
    k = 0
    while iters is None or k < iters:
        Xn = B + alpha * (PT @ X)
        k += 1
        d = float(np.abs(Xn - X).sum())
        X = Xn
        if tol is not None and d < tol:
            break
    return X, k
