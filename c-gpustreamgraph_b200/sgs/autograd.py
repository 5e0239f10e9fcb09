"""Weighted personalized PageRank as a differentiable torch op.

``personalized_pagerank(graph, w, T)`` returns X with
X = (1 - alpha) T + alpha P^T X, P[u, v] = w_uv / sum_v' w_uv', for every
column of T (the reference's PageRank fixed point,
samples/hybrid_pr/hybrid_pr.cu:26-151, with edge weights and teleport
vectors; T = 1 and unit weights give the reference's PageRank).  The
backward pass is the adjoint fixed point Y = dL/dX + alpha P Y solved by the
same CUDA kernels, then dL/dT = (1 - alpha) Y and the per-edge
dL/dw_uv = sum_k X[u,k] (alpha Y[v,k] - Y[u,k] + dL/dX[u,k]) / s_u.

Everything runs through the C ABI (``sgs_ppr_forward`` /
``sgs_ppr_backward``) on CUDA float64 tensors; float32 inputs are promoted
and their gradients returned as float32.
"""
from __future__ import annotations

import torch

from . import Ppr


class PersonalizedPageRank(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w, T, graph: Ppr, alpha: float, tol, max_iter: int):
        if not (w.is_cuda and T.is_cuda):
            raise ValueError("personalized_pagerank needs CUDA tensors")
        w64 = w.detach().to(torch.float64).contiguous()
        T64 = T.detach().to(torch.float64).reshape(graph.nv, -1).contiguous()
        X = graph.forward(w64, T64, alpha=alpha, tol=tol, max_iter=max_iter)
        ctx.graph, ctx.alpha, ctx.tol, ctx.max_iter = graph, alpha, tol, max_iter
        ctx.w_dtype, ctx.T_dtype, ctx.T_shape = w.dtype, T.dtype, T.shape
        ctx.save_for_backward(w64, X)
        return X

    @staticmethod
    def backward(ctx, gX):
        w64, X = ctx.saved_tensors
        need_w, need_T = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        if not (need_w or need_T):
            return None, None, None, None, None, None
        G = gX.detach().to(torch.float64).contiguous()
        gw, gT = ctx.graph.backward(w64, X, G, alpha=ctx.alpha, tol=ctx.tol,
                                    max_iter=ctx.max_iter, want_w=need_w, want_T=need_T)
        gw = gw.to(ctx.w_dtype) if need_w else None
        gT = gT.to(ctx.T_dtype).reshape(ctx.T_shape) if need_T else None
        return gw, gT, None, None, None, None


def personalized_pagerank(graph: Ppr, w: torch.Tensor, T: torch.Tensor, alpha: float = 0.85,
                          tol=None, max_iter: int = 100000) -> torch.Tensor:
    """X[nv, K] (float64) for edge weights w[ne] and teleport vectors T[nv, K]."""
    return PersonalizedPageRank.apply(w, T, graph, alpha, tol, max_iter)
