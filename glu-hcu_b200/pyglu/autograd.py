"""Differentiable sparse solve with a hand-written adjoint.

For x = A^{-1} b and a scalar loss L(x) with dL/dx = g:
    lambda = A^{-T} g                 (transposed solves with the stored factors,
                                       U^T then L^T, FP64-refined)
    dL/db  = lambda
    dL/dA_ij = -lambda_i x_j          (only on A's nonzero pattern)
The reference has no differentiation; this is new capability on top of its
factors and solves.
"""
from __future__ import annotations

import numpy as np


def _torch():
    import torch

    return torch


class _SparseSolve:
    _fn = None

    @classmethod
    def get(cls):
        if cls._fn is None:
            torch = _torch()

            class SparseSolveFunction(torch.autograd.Function):
                @staticmethod
                def forward(ctx, values, b, lu, tol, maxiter):
                    dev = b.device
                    v = values.detach().to(torch.float64)
                    lu._adj_version = getattr(lu, "_adj_version", 0) + 1
                    ver = lu._adj_version
                    if v.is_cuda:
                        lu.refactor_device(v.contiguous())
                        # the solve runs where the values are, whatever b's device
                        bb = b.detach().to(device=v.device, dtype=torch.float64).reshape(1, -1).contiguous()
                        x = torch.empty_like(bb)
                        lu.solve_device(bb, x, refine=True, tol=tol, maxiter=maxiter)
                        x = x.reshape(-1).to(dev)
                    else:
                        lu.refactor(v.cpu().numpy())
                        x = torch.from_numpy(
                            lu.solve(b.detach().cpu().numpy(), refine=True, tol=tol, maxiter=maxiter)).to(dev)
                    ctx.lu = lu
                    ctx.values_device = values.device
                    ctx.ver = ver
                    ctx.tol = tol
                    ctx.maxiter = maxiter
                    ctx.save_for_backward(v, x)
                    return x

                @staticmethod
                def backward(ctx, gx):
                    lu = ctx.lu
                    v, x = ctx.saved_tensors
                    if getattr(lu, "_adj_version", None) != ctx.ver:  # factors were replaced since
                        if v.is_cuda:
                            lu.refactor_device(v.contiguous())
                        else:
                            lu.refactor(v.cpu().numpy())
                        lu._adj_version = ctx.ver
                    g = gx.detach().to(torch.float64)
                    if v.is_cuda:
                        g = g.to(v.device)
                        gg = g.reshape(1, -1).contiguous()
                        lam = torch.empty_like(gg)
                        lu.solve_device(gg, lam, refine=True, tol=ctx.tol, maxiter=ctx.maxiter, trans="T")
                        lam = lam.reshape(-1)
                    else:
                        lam = torch.from_numpy(lu.solve(g.cpu().numpy(), refine=True, tol=ctx.tol,
                                                        maxiter=ctx.maxiter, trans="T"))
                    an = lu.analysis
                    rows = torch.as_tensor(an.ai.astype(np.int64), device=lam.device)
                    cols = torch.as_tensor(np.repeat(np.arange(an.n), np.diff(an.ap.astype(np.int64))),
                                           device=lam.device)
                    xx = x.to(lam.device)
                    gvals = -lam[rows] * xx[cols]
                    return gvals.to(ctx.values_device), lam.to(gx.device), None, None, None

            cls._fn = SparseSolveFunction
        return cls._fn


def sparse_solve(values, b, lu, tol=1e-12, maxiter=20):
    """x = A(values)^{-1} b, differentiable in ``values`` and ``b``.

    ``lu`` is a :class:`pyglu.GLUFactorization` of the pattern; ``values`` is a
    float64 tensor in the data order of that pattern (the CSC ``data`` array
    given to ``splu``).  The forward refactorizes with ``values`` and solves
    with FP64 refinement; the backward runs the adjoint transposed solves.
    """
    return _SparseSolve.get().apply(values, b, lu, tol, maxiter)
