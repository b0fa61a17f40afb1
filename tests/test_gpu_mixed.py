"""Mixed-precision CG with FP64 iterative refinement (FP32 and BF16 values)."""
import numpy as np
import pytest
import torch

from mpsparse_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bits,ir_mode", [(32, "replace"), (32, "restart"), (16, "auto")])
def test_ir_reaches_1e10(mps, oracle, bits, ir_mode):
    c = W.lognormal_diffusion_3d(32, 1.0, 4.0, 0)
    e = torch.empty(0)
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e, c.n, c.n)
    b = W.rhs(c.n, 1).astype(np.float64)
    x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
    info = A.cg_mixed(torch.from_numpy(b).cuda(), x, tol=1e-10, value_bits=bits, ir_mode=ir_mode)
    assert info["converged"] and info["rel_resid"] <= 1e-10
    Ao = oracle.Csr(*c.to_csr(), c.n)
    xr = x.cpu().numpy()
    assert oracle.true_residual(Ao, b, xr) <= 1.5e-10
    xo, io = oracle.cg(Ao, b, tol=1e-13, max_iter=20000)
    assert np.linalg.norm(xr - xo) / np.linalg.norm(xo) <= 1e-8


@pytest.mark.parametrize("precond", ["jacobi", "fsai"])
def test_reliable_updates_vs_restart(mps, oracle, precond):
    """Both refinement forms reach an FP64-checked 1e-6 on a log-normal
    system; reliable updates keep the Krylov space and need fewer FP32
    iterations than restarted sweeps."""
    c = W.lognormal_diffusion_2d(160, 120, 1.5, 8.0, 11)
    e = torch.empty(0)
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e, c.n, c.n)
    if precond == "fsai":
        from mpsparse_b200.fsai import LearnedFsai
        LearnedFsai.load().attach(A)
    Ao = oracle.Csr(*c.to_csr(), c.n)
    b = W.rhs(c.n, 3).astype(np.float64)
    its = {}
    for mode in ("replace", "restart"):
        x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
        info = A.cg_mixed(torch.from_numpy(b).cuda(), x, tol=1e-6, inner_tol=1e-3, max_inner=20000,
                          precond=precond, ir_mode=mode)
        assert info["converged"], mode
        assert oracle.true_residual(Ao, b, x.cpu().numpy()) <= 1e-6 * 1.01
        its[mode] = info["inner_iters"]
    assert its["replace"] <= its["restart"], its
    with pytest.raises(RuntimeError):
        A.cg_mixed(torch.from_numpy(b).cuda(), x, tol=1e-6, value_bits=16, ir_mode="replace")
