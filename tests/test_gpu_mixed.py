"""Mixed-precision CG with FP64 iterative refinement (FP32 and BF16 values)."""
import numpy as np
import pytest
import torch

from mpsparse_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bits", [32, 16])
def test_ir_reaches_1e10(mps, oracle, bits):
    c = W.lognormal_diffusion_3d(32, 1.0, 4.0, 0)
    e = torch.empty(0)
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e, c.n, c.n)
    b = W.rhs(c.n, 1).astype(np.float64)
    x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
    info = A.cg_mixed(torch.from_numpy(b).cuda(), x, tol=1e-10, value_bits=bits)
    assert info["converged"] and info["rel_resid"] <= 1e-10
    Ao = oracle.Csr(*c.to_csr(), c.n)
    xr = x.cpu().numpy()
    assert oracle.true_residual(Ao, b, xr) <= 1.5e-10
    xo, io = oracle.cg(Ao, b, tol=1e-13, max_iter=20000)
    assert np.linalg.norm(xr - xo) / np.linalg.norm(xo) <= 1e-8
