"""CSR SpMV on the GPU against the FP64 oracle (FP32 accumulation bound)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _make(mps, rp, ci, cv, n_rows, n_cols):
    rows = np.repeat(np.arange(n_rows, dtype=np.int64), np.diff(rp))
    keys = torch.from_numpy((rows << 32) | ci.astype(np.int64))
    vals = torch.from_numpy(cv.astype(np.float32))
    e = torch.empty(0)
    return mps.spmv.csr_tensor(keys, vals, e, e, e, n_rows, n_cols)


def _check(oracle, rp, ci, cv, n_rows, x, y):
    A = oracle.Csr(rp, ci, cv, n_rows)
    ref = oracle.spmv(A, x.astype(np.float64))
    bound = oracle.spmv(oracle.Csr(rp, ci, np.abs(cv), n_rows), np.abs(x).astype(np.float64))
    err = np.abs(y.astype(np.float64) - ref)
    assert np.all(err <= 1e-6 * bound + 1e-30), err.max()


def test_golden_laplacian(mps, golden, oracle):
    g = golden("laplacian12")
    n = int(g["n"])
    A = _make(mps, g["row_ptr"], g["col_ind"], g["csr_vals"], n, n)
    b = torch.zeros(n)
    A.mv(torch.from_numpy(g["x"]), b)
    assert np.allclose(b.numpy(), g["y"], rtol=1e-5, atol=1e-5)
    _check(oracle, g["row_ptr"], g["col_ind"], g["csr_vals"], n, g["x"], b.numpy())


@pytest.mark.parametrize("kind", ["c1", "graph", "longrows", "nonsquare", "emptyrows"])
def test_structures(mps, oracle, kind):
    from mpsparse_b200 import workloads as W
    rng = np.random.default_rng(0)
    if kind == "c1":
        c = W.laplacian_256()
        rp, ci, cv = c.to_csr(); nr = nc = c.n
    elif kind == "graph":
        c = W.graph_laplacian(50000, 8, 1)
        rp, ci, cv = c.to_csr(); nr = nc = c.n
    else:
        nr, nc = (20000, 20000) if kind != "nonsquare" else (7000, 300001)
        lens = rng.integers(0, 12, nr)
        if kind == "longrows":
            lens[5] = 150000; lens[777] = 9000; lens[778] = 2500; lens[-1] = 40000
        if kind == "emptyrows":
            lens[rng.random(nr) < 0.7] = 0
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
        ci = np.concatenate([np.sort(rng.choice(nc, l, replace=l > nc)) for l in lens]).astype(np.int32)
        cv = rng.standard_normal(rp[-1]).astype(np.float32)
    A = _make(mps, rp, ci, cv, nr, nc)
    x = rng.standard_normal(nc).astype(np.float32)
    y = torch.zeros(nr, device="cuda")
    A.mv(torch.from_numpy(x).cuda(), y)
    _check(oracle, rp, ci, cv, nr, x, y.cpu().numpy())


def test_mv_dot_deterministic(mps, oracle):
    from mpsparse_b200 import workloads as W
    c = W.lognormal_diffusion_2d(300, 200, 1.0, 8.0, 2)
    rp, ci, cv = c.to_csr()
    A = _make(mps, rp, ci, cv, c.n, c.n)
    rng = np.random.default_rng(1)
    x = torch.from_numpy(rng.standard_normal(c.n).astype(np.float32)).cuda()
    w = torch.from_numpy(rng.standard_normal(c.n).astype(np.float32)).cuda()
    y = torch.empty(c.n, device="cuda")
    d1 = A.mv_dot(x, w, y)
    d2 = A.mv_dot(x, w, y)
    assert d1 == d2                                    # bitwise run-to-run
    ref = float(w.double().cpu() @ y.double().cpu())
    assert abs(d1 - ref) <= 1e-12 * abs(ref) + 1e-9


def test_spmv_through_cabi(mps, golden):
    import ctypes as C
    from tests import cabi
    g = golden("laplacian12")
    n = int(g["n"])
    L = cabi.lib()
    h = C.c_void_p()
    k = torch.from_numpy(g["keys"]).cuda()
    v = torch.from_numpy(g["vals"]).cuda()
    cabi.check(L.mps_csr_create_from_keys(cabi.ptr(k), cabi.ptr(v), k.numel(), n, n, C.byref(h), None))
    x = torch.from_numpy(g["x"]).cuda()
    y = torch.empty(n, device="cuda")
    cabi.check(L.mps_csr_spmv(h, cabi.ptr(x), cabi.ptr(y), None))
    d = torch.empty(1, dtype=torch.float64, device="cuda")
    y2 = torch.empty(n, device="cuda")
    cabi.check(L.mps_csr_spmv_dot(h, cabi.ptr(x), cabi.ptr(x), cabi.ptr(y2), cabi.ptr(d), None))
    torch.cuda.synchronize()
    L.mps_csr_destroy(h)
    assert np.allclose(y.cpu().numpy(), g["y"], rtol=1e-5, atol=1e-5)
    assert torch.equal(y, y2)
    assert abs(d.item() - float(g["x"].astype(np.float64) @ g["y"])) < 1e-3


@pytest.mark.parametrize("kind", ["c1", "longrows", "emptyrows"])
def test_every_plan_variant(mps, oracle, kind):
    """Each tile plan the autotuner can pick (tile size, TMA pipeline depth,
    L2 hint) gives the same answer within the FP32 bound."""
    from mpsparse_b200 import workloads as W
    rng = np.random.default_rng(3)
    if kind == "c1":
        c = W.lognormal_diffusion_2d(200, 150, 1.0, 8.0, 4)
        rp, ci, cv = c.to_csr(); nr = nc = c.n
    else:
        nr = nc = 30000
        lens = rng.integers(0, 12, nr)
        if kind == "longrows":
            lens[9] = 70000; lens[1000] = 3000; lens[1001] = 2049
        else:
            lens[rng.random(nr) < 0.8] = 0
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
        ci = np.concatenate([np.sort(rng.choice(nc, l, replace=l > nc)) for l in lens]).astype(np.int32)
        cv = rng.standard_normal(rp[-1]).astype(np.float32)
    A = _make(mps, rp, ci, cv, nr, nc)
    x = rng.standard_normal(nc).astype(np.float32)
    xt = torch.from_numpy(x).cuda()
    for tile in (256, 0, 8192):
        for stages in (2, 3):
            for hint in (0, 1):
                A.set_plan(tile, stages, hint)
                y = torch.full((nr,), float("nan"), device="cuda")
                A.mv(xt, y)
                _check(oracle, rp, ci, cv, nr, x, y.cpu().numpy())
    with pytest.raises(RuntimeError):
        A.set_plan(0, 5, 0)


def test_autotune_then_solve(mps, oracle):
    from mpsparse_b200 import workloads as W
    from tests.helpers import assert_solved_fp32
    c = W.lognormal_diffusion_2d(128, 128, 1.0, 8.0, 5)
    rp, ci, cv = c.to_csr()
    A = _make(mps, rp, ci, cv, c.n, c.n)
    b = W.rhs(c.n, 1)
    x = torch.zeros(c.n, device="cuda")
    A.cgd(torch.from_numpy(b).float().cuda(), x, tol=1e-6, max_iter=5000)   # graph captured
    choice = A.autotune()
    assert choice["stages"] in (2, 3) and choice["evict_first"] in (0, 1)
    assert 256 <= choice["tile_nnz"] <= 8192 and choice["spmv_us"] > 0
    x.zero_()
    info = A.cgd(torch.from_numpy(b).float().cuda(), x, tol=1e-6, max_iter=5000)
    assert info["stop_rule_met"]
    assert_solved_fp32(oracle, oracle.Csr(rp, ci, cv, c.n), b, x.cpu().numpy(), 1e-6, info)


def test_sparse_csr_export(mps, oracle):
    """csr_tensor.sparse_csr(): the sorted matrix as a torch.sparse_csr_tensor
    whose arrays equal the handle's CSR and whose product matches A.mv."""
    from mpsparse_b200 import workloads as W
    c = W.lognormal_diffusion_2d(96, 80, 1.0, 6.0, 2).shuffled(3)
    e = torch.empty(0)
    A = mps.spmv.csr_tensor(torch.from_numpy(c.keys()), torch.from_numpy(c.vals), e, e, e, c.n, c.n)
    S = A.sparse_csr()
    assert S.layout == torch.sparse_csr and S.is_cuda and tuple(S.shape) == (c.n, c.n)
    rp, ci, cv = A.csr()
    assert torch.equal(S.crow_indices(), rp) and torch.equal(S.col_indices(), ci)
    assert torch.equal(S.values(), cv)
    orp, oci, ocv = oracle.coo_to_csr(c.keys(), c.vals, c.n, c.n)
    assert np.array_equal(rp.cpu().numpy(), orp) and np.array_equal(ci.cpu().numpy(), oci)
    x = torch.randn(c.n, device="cuda")
    y = torch.empty(c.n, device="cuda")
    A.mv(x, y)
    assert torch.allclose(S @ x, y, rtol=1e-5, atol=1e-5)
