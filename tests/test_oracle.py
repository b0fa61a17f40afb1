"""The CPU oracle against the golden fixtures and independent references."""
import numpy as np
import pytest


def test_sort_matches_torch_csr(golden, oracle):
    g = golden("laplacian12")
    rp, ci, cv = oracle.coo_to_csr(g["keys"], g["vals"], int(g["n"]), int(g["n"]))
    assert np.array_equal(rp, g["row_ptr"])
    assert np.array_equal(ci, g["col_ind"])
    assert np.array_equal(cv, g["csr_vals"])


def test_sort_duplicates_empty_rows_nonsquare(golden, oracle):
    g = golden("duplicates")
    rp, ci, cv = oracle.coo_to_csr(g["keys"], g["vals"], int(g["n_rows"]), int(g["n_cols"]))
    assert np.array_equal(rp, g["row_ptr"])
    assert np.array_equal(ci, g["col_ind"])
    assert np.array_equal(cv, g["csr_vals"])


def test_sort_matches_stable_argsort(oracle):
    rng = np.random.default_rng(3)
    n_rows, n_cols, nnz = 70000, 123457, 50000
    rows = rng.integers(0, n_rows, nnz)
    cols = rng.integers(0, n_cols, nnz)
    keys = (rows << 32) | cols
    keys[10:20] = keys[0]
    rows, cols = keys >> 32, keys & 0xFFFFFFFF
    vals = np.arange(nnz, dtype=np.float32)
    rp, ci, cv = oracle.coo_to_csr(keys, vals, n_rows, n_cols)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(cv, vals[order])
    assert np.array_equal(ci, cols[order])
    assert np.array_equal(rp, np.searchsorted(rows[order], np.arange(n_rows + 1)).astype(np.int32))


def test_sort_rejects_out_of_range(oracle):
    keys = np.array([(5 << 32) | 1], dtype=np.int64)
    with pytest.raises(ValueError):
        oracle.coo_to_csr(keys, np.ones(1, np.float32), 5, 5)


def test_sort_empty(oracle):
    rp, ci, cv = oracle.coo_to_csr(np.zeros(0, np.int64), np.zeros(0, np.float32), 4, 4)
    assert rp.tolist() == [0, 0, 0, 0, 0] and ci.size == 0


def test_spmv_matches_torch(golden, oracle):
    g = golden("laplacian12")
    A = oracle.Csr(g["row_ptr"], g["col_ind"], g["csr_vals"], int(g["n"]))
    assert np.allclose(oracle.spmv(A, g["x"]), g["y"], rtol=0, atol=1e-12)


def test_bcsr_spmv_matches_scipy(golden, oracle):
    g = golden("block16")
    A = oracle.Csr(g["row_ptr"], g["col_ind"], g["vals"], int(g["n"]), 4)
    assert np.allclose(oracle.spmv(A, g["x"]), g["y"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("k", [1, 2, 5, 10, 20])
def test_cg_iterates_match_scipy(golden, oracle, k):
    g = golden("laplacian12")
    A = oracle.Csr(g["row_ptr"], g["col_ind"], g["csr_vals"], int(g["n"]))
    x, info = oracle.cg(A, g["b"], tol=0.0, max_iter=k)
    ref = g["cg_iterates"][k - 1]
    assert np.linalg.norm(x - ref) <= 1e-12 * np.linalg.norm(ref)
    assert info["iters"] == k


@pytest.mark.parametrize("k", [1, 3, 8])
def test_bicgstab_iterates_match_scipy(golden, oracle, k):
    g = golden("block16")
    A = oracle.Csr(g["row_ptr"], g["col_ind"], g["vals"], int(g["n"]), 4)
    x, _ = oracle.bicgstab(A, g["b"], tol=0.0, max_iter=k)
    ref = g["bicgstab_iterates"][k - 1]
    assert np.linalg.norm(x - ref) <= 1e-12 * np.linalg.norm(ref)


def test_richardson_matches_loop(golden, oracle):
    g = golden("laplacian12")
    A = oracle.Csr(g["row_ptr"], g["col_ind"], g["csr_vals"], int(g["n"]))
    x, info = oracle.richardson(A, g["b"])
    assert info["iters"] == 1000
    assert np.abs(x - g["richardson_x"]).max() <= 1e-6


def test_compat_quirks(golden, oracle):
    """Reference stop rules: CG checks rr < 1e-5 every 50 iterations on the
    pre-update value; BiCGSTAB starts from rho0 = 1 + b.b."""
    g = golden("laplacian12")
    A = oracle.Csr(g["row_ptr"], g["col_ind"], g["csr_vals"], int(g["n"]))
    _, info = oracle.cg(A, g["b"], compat=True)
    assert info["iters"] % 50 == 1 and info["converged"]
    x1, _ = oracle.bicgstab(A, g["b"], compat=False, tol=0.0, max_iter=1)
    x2, _ = oracle.bicgstab(A, g["b"], compat=True)  # first iterate scaled by (1+bb)/bb
    assert not np.allclose(x1, x2)


def test_jacobi_pcg_converges(oracle):
    from mpsparse_b200 import workloads as W
    c = W.lognormal_diffusion_2d(32, 32, 1.5, 4.0, 0)
    rp, ci, cv = c.to_csr()
    A = oracle.Csr(rp, ci, cv, c.n)
    b = W.rhs(c.n, 1)
    _, i0 = oracle.cg(A, b, tol=1e-8, max_iter=5000)
    x, i1 = oracle.cg(A, b, tol=1e-8, max_iter=5000, precond="jacobi")
    assert i1["converged"] and i1["iters"] < i0["iters"]
    assert oracle.true_residual(A, b, x) < 1e-7
