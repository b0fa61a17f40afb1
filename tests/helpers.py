"""Shared checks for the GPU tests."""
import numpy as np

EPS32 = 2.0 ** -24


def fp32_floor(oracle, A, b, x, factor=16.0):
    """Attainable FP64-checked residual of an FP32 solution vector:
    factor * eps32 * || |A| |x| || / ||b|| (componentwise rounding bound of
    b - A fl32(x), times a margin for the rounding accumulated by the solver)."""
    Aabs = oracle.Csr(A.row_ptr, A.col_ind, np.abs(A.val), A.n, A.block)
    return factor * EPS32 * np.linalg.norm(oracle.spmv(Aabs, np.abs(x))) / np.linalg.norm(b)


def assert_solved_fp32(oracle, A, b, x, tol, info=None, floor_factor=16.0):
    """Final FP32 answer checked by the FP64 true residual: below 2*tol, or at
    the FP32 rounding floor when that floor is above it.  With the solver's
    info dict: its true_resid (recomputed on the GPU in FP64) equals the
    oracle's FP64 true residual of the same x, and `converged` says exactly
    whether that residual meets tol."""
    x = np.asarray(x, dtype=np.float64)
    res = oracle.true_residual(A, b, x)
    bound = max(2.0 * tol, fp32_floor(oracle, A, b, x, floor_factor))
    assert res <= bound, (res, bound)
    if info is not None:
        assert abs(info["true_resid"] - res) <= 1e-6 * res + 1e-30, (info["true_resid"], res)
        assert info["converged"] == (info["true_resid"] <= tol), info
    return res
