"""Differentiable solve against dense float64 torch.linalg.solve gradients.

Tolerance: 1e-3 relative in 2-norm (FP32 solves to tol 1e-7 on well
conditioned systems; the forward and both gradients inherit that error)."""
import numpy as np
import pytest
import torch

from mpsparse_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _dense(rp, ci, v, n):
    A = torch.zeros(n, n, dtype=torch.float64)
    rows = np.repeat(np.arange(n), np.diff(rp))
    A[rows, ci] = torch.from_numpy(v.astype(np.float64))
    return A


def _rel(a, b):
    return float((a.double().cpu() - b).norm() / b.norm())


@pytest.mark.parametrize("method", ["cg", "bicgstab"])
def test_gradients_match_dense(mps, method):
    from mpsparse_b200.autograd import sparse_solve
    if method == "cg":
        c = W.lognormal_diffusion_2d(20, 15, 0.5, 3.0, 1)
        rp, ci, v = c.to_csr()
        n = c.n
    else:
        blk = W.block_dominant(32, 3, seed=2, block=4)
        c = blk.to_coo()
        rp, ci, v = c.to_csr()
        n = c.n
    rng = np.random.default_rng(0)
    b = rng.standard_normal(n)
    gout = rng.standard_normal(n)
    vals = torch.tensor(v, device="cuda", dtype=torch.float32, requires_grad=True)
    bt = torch.tensor(b, device="cuda", dtype=torch.float32, requires_grad=True)
    x = sparse_solve(torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), vals, bt, method=method,
                     tol=1e-7)
    (x * torch.tensor(gout, device="cuda", dtype=torch.float32)).sum().backward()
    # dense reference in float64
    Ad = _dense(rp, ci, v, n).requires_grad_(True)
    bd = torch.tensor(b, dtype=torch.float64, requires_grad=True)
    xd = torch.linalg.solve(Ad, bd)
    (xd * torch.tensor(gout)).sum().backward()
    rows = np.repeat(np.arange(n), np.diff(rp))
    gA = Ad.grad[rows, ci]
    assert _rel(x.detach(), xd.detach()) <= 1e-3
    assert _rel(bt.grad, bd.grad) <= 1e-3
    assert _rel(vals.grad, gA) <= 1e-3
