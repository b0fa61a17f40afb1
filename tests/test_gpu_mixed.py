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


def test_fsai_graph_matches_host_loop(mps, oracle):
    """The FSAI-PCG body fuses the x/r update into the G-apply and runs the
    residual replacement under a graph IF node; launching the same kernels
    from the host (where the replacement kernels return at once unless due)
    must give bit-identical results, for reliable updates and plain FP32."""
    from mpsparse_b200.fsai import LearnedFsai
    c = W.lognormal_diffusion_2d(160, 120, 1.5, 8.0, 21)
    e = torch.empty(0)
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e, c.n, c.n)
    LearnedFsai.load().attach(A)
    A.set_persistent(False)            # the graph form (the persistent one: test_gpu_persistent)
    b = torch.from_numpy(W.rhs(c.n, 4).astype(np.float64)).cuda()
    xs, infos = [], []
    for host_loop in (False, True):
        x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
        infos.append(A.cg_mixed(b, x, tol=1e-9, inner_tol=1e-3, max_inner=20000, precond="fsai",
                                ir_mode="replace", host_loop=host_loop))
        xs.append(x)
    assert infos[0] == infos[1]
    assert infos[0]["converged"] and infos[0]["outer_iters"] >= 2
    assert torch.equal(xs[0], xs[1])
    Ao = oracle.Csr(*c.to_csr(), c.n)
    assert oracle.true_residual(Ao, b.cpu().numpy(), xs[0].cpu().numpy()) <= 1e-9 * 1.01
    x32 = []
    for host_loop in (False, True):
        x = torch.zeros(c.n, device="cuda")
        i = A.cgd(b.float(), x, tol=1e-6, max_iter=20000, precond="fsai", host_loop=host_loop)
        assert i["stop_rule_met"]
        x32.append((x, i))
    assert x32[0][1] == x32[1][1] and torch.equal(x32[0][0], x32[1][0])


def test_fsai_stall_fallback_graph_matches_host_loop(mps):
    """A poor factor trips the stall watch: the direction restarts from
    D^-1 r, read from the current buffer of the residual pair."""
    c = W.lognormal_diffusion_2d(64, 64, 1.5, 8.0, 7)
    e = torch.empty(0)
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e, c.n, c.n)
    n = c.n
    rp, ci, _ = c.to_csr()
    rows_all = np.repeat(np.arange(n), np.diff(rp))
    keep = ci <= rows_all
    rows = rows_all[keep]
    gci = ci[keep]
    gv = np.where(gci == rows, 1.0, 5.0 * np.random.default_rng(0).standard_normal(keep.sum()))
    grp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int32)
    A.set_fsai(torch.from_numpy(grp), torch.from_numpy(gci.astype(np.int32)),
               torch.from_numpy(gv.astype(np.float32)))
    b = torch.from_numpy(W.rhs(n, 1)).cuda()
    out = []
    for host_loop in (False, True):
        x = torch.zeros(n, device="cuda")
        info = A.cgd(b, x, tol=1e-6, max_iter=20000, precond="fsai", stall_window=20,
                     host_loop=host_loop)
        assert info["stalled"] and info["stop_rule_met"]
        out.append((x, info))
    assert out[0][1] == out[1][1] and torch.equal(out[0][0], out[1][0])


@pytest.mark.parametrize("precond", ["none", "jacobi", "fsai"])
def test_mixed_zero_and_nonfinite_rhs(mps, precond):
    """b = 0 stops at once with x = 0; a NaN in b is reported, not iterated
    on (both settled on the device, read back with the result)."""
    c = W.lognormal_diffusion_2d(48, 40, 1.0, 4.0, 2)
    e = torch.empty(0)
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e, c.n, c.n)
    if precond == "fsai":
        from mpsparse_b200.fsai import LearnedFsai
        LearnedFsai.load().attach(A)
    x = torch.full((c.n,), 7.0, dtype=torch.float64, device="cuda")
    info = A.cg_mixed(torch.zeros(c.n, dtype=torch.float64, device="cuda"), x, tol=1e-8, precond=precond)
    assert info["converged"] and info["rel_resid"] == 0.0 and info["inner_iters"] == 0
    assert torch.count_nonzero(x) == 0
    b = torch.from_numpy(W.rhs(c.n, 2)).double().cuda()
    b[c.n // 2] = float("nan")
    with pytest.raises(RuntimeError, match="NaN|non-finite|Inf"):
        A.cg_mixed(b, x, tol=1e-8, precond=precond)
    # the handle stays usable
    b[c.n // 2] = 1.0
    info = A.cg_mixed(b, x, tol=1e-8, precond=precond)
    assert info["converged"]


def test_bf16_default_inner_tol(mps, oracle):
    """BF16 values: the default sweep target (0.1) reaches 1e-10 with fewer
    FP32 iterations than asking each sweep for 1e-3, which a BF16-valued
    operator (about 2^-9 relative from A) cannot deliver without many
    wasted iterations."""
    c = W.lognormal_diffusion_3d(48, 1.0, 8.0, 2)
    e = torch.empty(0)
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e, c.n, c.n)
    b = torch.from_numpy(W.rhs(c.n, 4).astype(np.float64)).cuda()
    x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
    dflt = A.cg_mixed(b, x, tol=1e-10, value_bits=16)
    assert dflt["converged"] and dflt["rel_resid"] <= 1e-10
    Ao = oracle.Csr(*c.to_csr(), c.n)
    assert oracle.true_residual(Ao, b.cpu().numpy(), x.cpu().numpy()) <= 1.5e-10
    x.zero_()
    tight = A.cg_mixed(b, x, tol=1e-10, value_bits=16, inner_tol=1e-3, max_inner=20000, max_outer=200)
    assert tight["converged"]
    assert dflt["inner_iters"] < tight["inner_iters"], (dflt, tight)
