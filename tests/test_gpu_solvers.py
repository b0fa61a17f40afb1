"""CG / PCG / BiCGSTAB / Richardson on the GPU against the FP64 oracle.

Tolerance (from the solver contract): each of the first 20 FP32 iterates is
within 1e-5 relative (2-norm) of the FP64 transcription; final answers are
checked by the FP64 true residual ||b - A x|| / ||b||."""
import numpy as np
import pytest
import torch

from mpsparse_b200 import workloads as W
from tests.helpers import assert_solved_fp32

pytestmark = pytest.mark.gpu
ITERATE_RTOL = 1e-5
NO_TOL = 1e-300


def _csr_tensor(mps, coo):
    e = torch.empty(0)
    return mps.spmv.csr_tensor(torch.from_numpy(coo.keys()), torch.from_numpy(coo.vals), e, e, e,
                               coo.n, coo.n)


def _oracle_A(oracle, coo):
    return oracle.Csr(*coo.to_csr(), coo.n)


@pytest.fixture(scope="module")
def c1():
    return W.laplacian_256().shuffled(0)


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_cg_first_20_iterates(mps, oracle, c1):
    A = _csr_tensor(mps, c1)
    Ao = _oracle_A(oracle, c1)
    b = W.rhs(c1.n, 0)
    bt = torch.from_numpy(b).cuda()
    for k in range(1, 21):
        x = torch.zeros(c1.n, device="cuda")
        info = A.cgd(bt, x, tol=NO_TOL, max_iter=k)
        assert info["iters"] == k
        xo, _ = oracle.cg(Ao, b, tol=0.0, max_iter=k)
        assert _rel(x.cpu().numpy().astype(np.float64), xo) <= ITERATE_RTOL, k


def test_cg_converges_true_residual(mps, oracle, c1):
    A = _csr_tensor(mps, c1)
    Ao = _oracle_A(oracle, c1)
    b = W.rhs(c1.n, 0)
    x = torch.zeros(c1.n)
    info = A.cgd(torch.from_numpy(b), x, tol=1e-6, max_iter=2000)   # CPU tensors: drop-in path
    _, io = oracle.cg(Ao, b, tol=1e-6, max_iter=2000)
    assert info["stop_rule_met"] and abs(info["iters"] - io["iters"]) <= 5
    assert_solved_fp32(oracle, Ao, b, x.numpy(), 1e-6, info)


def test_cg_graph_host_loop_and_reruns_bitwise(mps, c1):
    A = _csr_tensor(mps, c1)
    A.set_persistent(False)            # the graph form (the persistent one: test_gpu_persistent)
    b = torch.from_numpy(W.rhs(c1.n, 3)).cuda()
    xs = []
    for host_loop in (False, True, False):
        x = torch.zeros(c1.n, device="cuda")
        info = A.cgd(b, x, tol=1e-6, host_loop=host_loop)
        xs.append((x.clone(), info["iters"]))
    assert xs[0][1] == xs[1][1] == xs[2][1]
    assert torch.equal(xs[0][0], xs[1][0]) and torch.equal(xs[0][0], xs[2][0])


def test_cg_reference_compat(mps, oracle, c1):
    A = _csr_tensor(mps, c1)
    Ao = _oracle_A(oracle, c1)
    b = W.rhs(c1.n, 5)
    x = torch.zeros(c1.n)
    info = A.cgd(torch.from_numpy(b), x, reference_compat=True)
    xo, io = oracle.cg(Ao, b, compat=True)
    assert info["iters"] == io["iters"] and info["iters"] % 50 == 1
    assert _rel(x.numpy().astype(np.float64), xo) <= 1e-4


def test_jacobi_pcg_iterates(mps, oracle):
    c = W.lognormal_diffusion_2d(64, 48, 1.5, 6.0, 7)
    A = _csr_tensor(mps, c)
    Ao = _oracle_A(oracle, c)
    b = W.rhs(c.n, 1)
    bt = torch.from_numpy(b).cuda()
    for k in (1, 2, 5, 10, 20):
        x = torch.zeros(c.n, device="cuda")
        A.cgd(bt, x, tol=NO_TOL, max_iter=k, precond="jacobi")
        xo, _ = oracle.cg(Ao, b, tol=0.0, max_iter=k, precond="jacobi")
        assert _rel(x.cpu().numpy().astype(np.float64), xo) <= ITERATE_RTOL, k
    x = torch.zeros(c.n, device="cuda")
    info = A.cgd(bt, x, tol=1e-6, max_iter=5000, precond="jacobi")
    info0 = A.cgd(bt, torch.zeros(c.n, device="cuda"), tol=1e-6, max_iter=5000)
    assert info["stop_rule_met"] and info["iters"] < info0["iters"]
    assert_solved_fp32(oracle, Ao, b, x.cpu().numpy(), 1e-6, info)


def test_bicgstab_iterates(mps, oracle):
    bm = W.block_dominant(256, 8, seed=2)
    c = bm.to_coo(drop_zeros=False)
    A = _csr_tensor(mps, c)
    Ao = _oracle_A(oracle, c)
    b = W.rhs(c.n, 2)
    bt = torch.from_numpy(b).cuda()
    for k in range(1, 21):
        x = torch.zeros(c.n, device="cuda")
        A.bicgstab(bt, x, tol=NO_TOL, max_iter=k)
        xo, io = oracle.bicgstab(Ao, b, tol=0.0, max_iter=k)
        assert _rel(x.cpu().numpy().astype(np.float64), xo) <= ITERATE_RTOL, k
    x = torch.zeros(c.n, device="cuda")
    info = A.bicgstab(bt, x, tol=1e-6)
    assert info["stop_rule_met"]
    assert_solved_fp32(oracle, Ao, b, x.cpu().numpy(), 1e-6, info)


def test_bicgstab_golden_scipy(mps, golden):
    g = golden("block16")
    rp, ci, v = g["row_ptr"], g["col_ind"], g["vals"]
    bm = W.Bcsr(rp, ci, v, 4, int(g["n"]))
    c = bm.to_coo(drop_zeros=False)
    A = _csr_tensor(mps, c)
    bt = torch.from_numpy(g["b"]).cuda()
    for k in range(1, 9):
        x = torch.zeros(c.n, device="cuda")
        A.bicgstab(bt, x, tol=NO_TOL, max_iter=k)
        ref = g["bicgstab_iterates"][k - 1]
        assert _rel(x.cpu().numpy().astype(np.float64), ref) <= ITERATE_RTOL


def test_bicgstab_reference_compat(mps, oracle, c1):
    """Delayed stop on the staged ||r||^2 (spmv.cpp:835-859) with rho0 = 1 + b.b.
    A well-conditioned system keeps FP32 and FP64 on the same side of the
    absolute 1e-5 threshold at every check."""
    bm = W.block_dominant(256, 8, seed=4)
    c = bm.to_coo(drop_zeros=False)
    A = _csr_tensor(mps, c)
    Ao = _oracle_A(oracle, c)
    b = W.rhs(c.n, 9)
    x = torch.zeros(c.n)
    info = A.bicgstab(torch.from_numpy(b), x, reference_compat=True)
    xo, io = oracle.bicgstab(Ao, b, compat=True)
    assert info["iters"] == io["iters"] == 51
    assert info["compat_snapshot"] and io["converged"]
    assert _rel(x.numpy().astype(np.float64), xo) <= 1e-5
    # C1: the cap and checkpoint path agree on iteration counts to a check
    x = torch.zeros(c1.n)
    info = _csr_tensor(mps, c1).bicgstab(torch.from_numpy(W.rhs(c1.n, 9)), x,
                                         reference_compat=True)
    assert info["iters"] % 50 == 1


def test_richardson(mps, oracle, golden, c1):
    g = golden("laplacian12")
    n = int(g["n"])
    e = torch.empty(0)
    A = mps.spmv.csr_tensor(torch.from_numpy(g["keys"]), torch.from_numpy(g["vals"]), e, e, e, n, n)
    x = torch.zeros(n)
    info = A.richardson(torch.from_numpy(g["b"]), x, reference_compat=True)
    assert info["iters"] == 1000
    assert _rel(x.numpy().astype(np.float64), g["richardson_x"]) <= ITERATE_RTOL
    A1 = _csr_tensor(mps, c1)
    b = W.rhs(c1.n, 4)
    x = torch.zeros(c1.n)
    A1.richardson(torch.from_numpy(b), x, omega=0.2, iters=301)      # odd count: ping-pong parity
    xo, _ = oracle.richardson(_oracle_A(oracle, c1), b, compat=False, omega=0.2, iters=301)
    assert _rel(x.numpy().astype(np.float64), xo) <= ITERATE_RTOL
    x2 = torch.zeros(c1.n)
    A1.iter_solve(torch.from_numpy(b), x2)                             # CG alias
    assert_solved_fp32(oracle, _oracle_A(oracle, c1), b, x2.numpy(), 1e-6)


def test_edge_cases(mps, c1):
    A = _csr_tensor(mps, c1)
    x = torch.ones(c1.n, device="cuda")
    info = A.cgd(torch.zeros(c1.n, device="cuda"), x)
    assert info["converged"] and info["iters"] == 0 and float(x.abs().max()) == 0.0
    assert info["true_resid"] == 0.0
    b = torch.ones(c1.n, device="cuda")
    b[17] = float("nan")
    with pytest.raises(RuntimeError, match="non-finite"):
        A.cgd(b, x)
    info = A.cgd(torch.ones(c1.n, device="cuda"), x, max_iter=3, tol=NO_TOL)   # still usable
    assert info["iters"] == 3
