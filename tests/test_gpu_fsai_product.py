"""FSAI preconditioner applied as one SpMV with M = G^T G (the product form):
M against an FP64 SciPy product of the factor, exact symmetry, the choice of
form, and PCG in product form against the split form (G then G^T) and
against its own host-launched loop."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from mpsparse_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _system(mps, c):
    e = torch.empty(0)
    return mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e, c.n, c.n)


def _learned(mps, nx, ny, seed):
    from mpsparse_b200.fsai import LearnedFsai
    c = W.lognormal_diffusion_2d(nx, ny, 1.5, 8.0, seed)
    A = _system(mps, c)
    LearnedFsai.load().attach(A)
    return c, A


def test_product_is_gtg(mps):
    c, A = _learned(mps, 96, 80, 3)
    assert A.fsai_apply()["form"] == "product"       # auto: small 2D system
    _, grp, gci = A.fsai_features()
    gv = A.fsai_g_values().cpu().numpy().astype(np.float64)
    grp, gci = grp.cpu().numpy().copy(), gci.cpu().numpy().copy()
    G = sp.csr_matrix((gv, gci, grp), shape=(c.n, c.n))
    Gs = sp.csr_matrix((np.ones_like(gv), gci, grp), shape=(c.n, c.n))
    P = (Gs.T @ Gs).tocsr()                             # pattern (no cancellation)
    P.sort_indices()
    rp, ci, v = (t.cpu().numpy().copy() for t in A.fsai_product())   # own their memory
    assert A.fsai_apply()["nnz_m"] == P.nnz == ci.size
    assert np.array_equal(rp, P.indptr) and np.array_equal(ci, P.indices)
    rows = np.repeat(np.arange(c.n), np.diff(rp))
    ref = np.asarray((G.T @ G).tocsr()[rows, ci]).ravel()
    scale = np.abs(ref).max()
    assert np.all(np.abs(v - ref) <= 2e-7 * np.abs(ref) + 1e-9 * scale)
    M = sp.csr_matrix((v, ci, rp), shape=(c.n, c.n))
    assert (M - M.T).count_nonzero() == 0               # exactly symmetric


def test_product_and_split_reach_the_same_solution(mps, oracle):
    c, A = _learned(mps, 160, 120, 21)
    b = torch.from_numpy(W.rhs(c.n, 4).astype(np.float64)).cuda()
    Ao = oracle.Csr(*c.to_csr(), c.n)
    res = {}
    for form in ("product", "split"):
        A.set_fsai_apply(form)
        assert A.fsai_apply()["form"] == form
        x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
        info = A.cg_mixed(b, x, tol=1e-9, inner_tol=1e-3, max_inner=20000, precond="fsai")
        assert info["converged"]
        assert oracle.true_residual(Ao, b.cpu().numpy(), x.cpu().numpy()) <= 1e-9 * 1.01
        res[form] = (x.cpu().numpy(), info["inner_iters"])
    xp, ip = res["product"]
    xs, is_ = res["split"]
    assert abs(ip - is_) <= max(3, 0.03 * is_), (ip, is_)
    assert np.linalg.norm(xp - xs) / np.linalg.norm(xs) <= 1e-7


def test_product_graph_matches_host_loop(mps):
    c, A = _learned(mps, 160, 120, 22)
    A.set_fsai_apply("product")
    A.set_persistent(False)            # the graph form (the persistent one: test_gpu_persistent)
    b = torch.from_numpy(W.rhs(c.n, 5).astype(np.float64)).cuda()
    xs, infos = [], []
    for host_loop in (False, True):
        x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
        infos.append(A.cg_mixed(b, x, tol=1e-9, inner_tol=1e-3, max_inner=20000, precond="fsai",
                                ir_mode="replace", host_loop=host_loop))
        xs.append(x)
    assert infos[0] == infos[1] and infos[0]["outer_iters"] >= 2
    assert torch.equal(xs[0], xs[1])
    out = []
    for host_loop in (False, True):
        x = torch.zeros(c.n, device="cuda")
        info = A.cgd(b.float(), x, tol=1e-6, max_iter=20000, precond="fsai", host_loop=host_loop)
        assert info["stop_rule_met"]
        out.append((x, info))
    assert out[0][1] == out[1][1] and torch.equal(out[0][0], out[1][0])
    # the restarted refinement runs the same product-form inner solve
    x = torch.zeros(c.n, dtype=torch.float64, device="cuda")
    info = A.cg_mixed(b, x, tol=1e-9, inner_tol=1e-3, max_inner=20000, precond="fsai", ir_mode="restart")
    assert info["converged"]


def test_product_stall_fallback(mps):
    c = W.lognormal_diffusion_2d(64, 64, 1.5, 8.0, 7)
    A = _system(mps, c)
    n = c.n
    rp, ci, _ = c.to_csr()
    rows_all = np.repeat(np.arange(n), np.diff(rp))
    keep = ci <= rows_all
    rows, gci = rows_all[keep], ci[keep]
    gv = np.where(gci == rows, 1.0, 5.0 * np.random.default_rng(0).standard_normal(keep.sum()))
    grp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int32)
    A.set_fsai_apply("product")
    A.set_fsai(torch.from_numpy(grp), torch.from_numpy(gci.astype(np.int32)),
               torch.from_numpy(gv.astype(np.float32)))
    assert A.fsai_apply()["form"] == "product"
    b = torch.from_numpy(W.rhs(n, 1)).cuda()
    out = []
    for host_loop in (False, True):
        x = torch.zeros(n, device="cuda")
        info = A.cgd(b, x, tol=1e-6, max_iter=20000, precond="fsai", stall_window=20,
                     host_loop=host_loop)
        assert info["stalled"] and info["stop_rule_met"]
        out.append((x, info))
    assert out[0][1] == out[1][1] and torch.equal(out[0][0], out[1][0])


def test_auto_keeps_split_for_large_3d(mps):
    """100^3 7-point: M would add 8 nonzeros per row over G and G^T (8M in
    all), more than one saved launch is worth; auto keeps the split form."""
    c = W.lognormal_diffusion_3d(100, 1.0, 4.0, 0)
    A = _system(mps, c)
    rp, ci, cv = c.to_csr()
    n = c.n
    rows_all = np.repeat(np.arange(n), np.diff(rp))
    keep = ci <= rows_all
    rows, gci = rows_all[keep], ci[keep]
    diag = cv[ci == rows_all]
    gv = np.where(gci == rows, 1.0 / np.sqrt(diag[rows]), 0.0).astype(np.float32)
    grp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int32)
    A.set_fsai(torch.from_numpy(grp), torch.from_numpy(gci.astype(np.int32)), torch.from_numpy(gv))
    assert A.fsai_apply() == {"form": "split", "nnz_m": 0}
    A.set_fsai_apply("product")
    f = A.fsai_apply()
    assert f["form"] == "product" and f["nnz_m"] > 2 * gci.size
    A.set_fsai_apply("split")
    assert A.fsai_apply()["form"] == "split"
