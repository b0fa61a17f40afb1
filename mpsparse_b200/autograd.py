"""Differentiable sparse solve: x = A^{-1} b with gradients for b and A.

The reference's sparse-QR bridge exposes a torch.autograd layer around its
direct solver (sparse_bridge/SPQR_layer.py:12-58).  This is the same layer
around the iterative solvers of this package:

* forward: x = A^{-1} b by CG (symmetric positive definite A) or BiCGSTAB;
* backward: lam = A^{-T} g (the adjoint solve, by the same solver on A^T,
  which for CG is A itself), then grad_b = lam and, on A's sparsity pattern,
  grad_A[k] = -lam[row_k] * x[col_k].

A is given in CSR form (row_ptr, col_ind, values); the values may require
grad.  Solves run in FP32 on the GPU; the gradients are as accurate as the
two solves (tol).
"""
from __future__ import annotations

import torch

from ._C import csr_tensor


def _handle(row_ptr, col_ind, values, n, transpose=False):
    rows = torch.repeat_interleave(torch.arange(n, device=row_ptr.device, dtype=torch.int64),
                                   (row_ptr[1:] - row_ptr[:-1]).to(torch.int64))
    cols = col_ind.to(torch.int64)
    if transpose:
        rows, cols = cols, rows
    keys = (rows << 32) | cols
    e = torch.empty(0)
    return csr_tensor(keys, values.detach().float(), e, e, e, n, n, fill_outputs=False)


def _solve(H, b, method, tol, max_iter, precond):
    x = torch.zeros(b.numel(), device=b.device, dtype=torch.float32)
    if method == "cg":
        info = H.cgd(b.float().contiguous(), x, tol=tol, max_iter=max_iter, precond=precond)
    else:
        info = H.bicgstab(b.float().contiguous(), x, tol=tol, max_iter=max_iter)
    # the FP32 solver's own stop test; the FP64 true residual of an FP32 x can
    # sit above tol on ill-conditioned systems (info["true_resid"])
    if not info["stop_rule_met"]:
        raise RuntimeError(f"sparse solve did not converge ({method}, {info['iters']} iterations)")
    return x


class SparseSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, row_ptr, col_ind, values, b, method="cg", tol=1e-6, max_iter=10000,
                precond="none"):
        n = row_ptr.numel() - 1
        H = _handle(row_ptr, col_ind, values, n)
        x = _solve(H, b, method, tol, max_iter, precond)
        ctx.save_for_backward(row_ptr, col_ind, values, x)
        ctx.H = H
        ctx.opts = (method, tol, max_iter, precond)
        return x.to(b.dtype)

    @staticmethod
    def backward(ctx, g):
        row_ptr, col_ind, values, x = ctx.saved_tensors
        method, tol, max_iter, precond = ctx.opts
        n = row_ptr.numel() - 1
        # adjoint solve A^T lam = g (A itself for CG)
        HT = ctx.H if method == "cg" else _handle(row_ptr, col_ind, values, n, transpose=True)
        lam = _solve(HT, g.contiguous(), method, tol, max_iter, precond if method == "cg" else "none")
        grad_values = None
        if ctx.needs_input_grad[2]:
            rows = torch.repeat_interleave(torch.arange(n, device=row_ptr.device),
                                           (row_ptr[1:] - row_ptr[:-1]).to(torch.int64))
            grad_values = (-lam[rows] * x[col_ind.long()]).to(values.dtype)
        grad_b = lam.to(g.dtype) if ctx.needs_input_grad[3] else None
        return None, None, grad_values, grad_b, None, None, None, None


def sparse_solve(row_ptr, col_ind, values, b, method="cg", tol=1e-6, max_iter=10000,
                 precond="none"):
    """x = A^{-1} b, differentiable in `values` and `b` (CUDA tensors)."""
    if method not in ("cg", "bicgstab"):
        raise ValueError("method must be 'cg' or 'bicgstab'")
    return SparseSolve.apply(row_ptr, col_ind, values, b, method, tol, max_iter, precond)
