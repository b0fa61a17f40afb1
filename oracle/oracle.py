"""ctypes front-end of the CPU oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Imported by tests/,
by ``__graft_entry__.smoke()`` and by ``bench.py``'s CPU-baseline leg; the
product package never imports it.

Parity status: sort/CSR and SpMV are pinned by golden fixtures generated from
the reference's own ground-truth checks (torch ``to_sparse_csr`` and torch
CSR ``mm``); solver iterates are pinned against scipy's CG/BiCGSTAB iterates.
The reference_compat quirks (iterative/BiCGSTAB/spmv.cpp, bicgstab.metal) are
restated from the source and are "parity unpinned": the reference runs only
on Metal.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    """Compile oracle.c with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


class _Opts(C.Structure):
    _fields_ = [("compat", C.c_int), ("max_iter", C.c_int), ("tol", C.c_double),
                ("omega", C.c_double), ("threads", C.c_int), ("precond", C.c_int)]


class _Info(C.Structure):
    _fields_ = [("iters", C.c_int), ("converged", C.c_int), ("breakdown", C.c_int),
                ("rel_resid", C.c_double)]


class _Op(C.Structure):
    _fields_ = [("row_ptr", C.c_void_p), ("col_ind", C.c_void_p), ("val", C.c_void_p),
                ("n", C.c_int64), ("block", C.c_int)]


def _declare(L):
    vp, i64, u64, u32 = C.c_void_p, C.c_int64, C.c_uint64, C.c_uint32
    L.orc_coo_to_csr.argtypes = [vp, vp, u64, u32, u32, vp, vp, vp]
    L.orc_coo_to_csr.restype = C.c_int
    L.orc_csr_spmv.argtypes = [vp, vp, vp, i64, vp, vp, C.c_int]
    L.orc_bcsr_spmv.argtypes = [vp, vp, vp, i64, C.c_int, vp, vp]
    for name in ("orc_cg", "orc_bicgstab", "orc_richardson"):
        f = getattr(L, name)
        f.argtypes = [C.POINTER(_Op), vp, vp, C.POINTER(_Opts), C.POINTER(_Info)]
        f.restype = C.c_int
    L.orc_true_residual.argtypes = [C.POINTER(_Op), vp, vp]
    L.orc_true_residual.restype = C.c_double
    L.orc_fsai_pattern.argtypes = [C.POINTER(_Op), vp, vp, vp, vp]
    L.orc_fsai_pattern.restype = C.c_int64
    L.orc_fsai_features.argtypes = [C.POINTER(_Op), C.c_int64, vp, vp, vp, vp]
    L.orc_mlp_forward.argtypes = [vp, vp, C.c_int64, vp]
    L.orc_mlp_backward.argtypes = [vp, vp, C.c_int64, vp, vp]
    L.orc_fsai_probe_loss_grad.argtypes = [C.POINTER(_Op), C.POINTER(_Op), vp, C.c_int, vp]
    L.orc_fsai_probe_loss_grad.restype = C.c_double


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


@dataclass
class Csr:
    """A CSR (block=0) or BCSR (block=B) matrix held as numpy arrays."""
    row_ptr: np.ndarray
    col_ind: np.ndarray
    val: np.ndarray
    n: int                 # scalar rows (= cols; square systems)
    block: int = 0

    def __post_init__(self):
        self.row_ptr = np.ascontiguousarray(self.row_ptr, dtype=np.int32)
        self.col_ind = np.ascontiguousarray(self.col_ind, dtype=np.int32)
        self.val = np.ascontiguousarray(self.val, dtype=np.float32)

    def _op(self) -> _Op:
        return _Op(_p(self.row_ptr).value, _p(self.col_ind).value, _p(self.val).value,
                   int(self.n), int(self.block))


def coo_to_csr(keys: np.ndarray, vals: np.ndarray, n_rows: int, n_cols: int):
    """Masked 4-bit LSD sort + compress + fixer; returns (row_ptr, col_ind, vals)."""
    keys = np.ascontiguousarray(keys).view(np.uint64)
    vals = np.ascontiguousarray(vals, dtype=np.float32)
    nnz = keys.shape[0]
    rp = np.empty(n_rows + 1, np.int32)
    ci = np.empty(max(nnz, 1), np.int32)
    ov = np.empty(max(nnz, 1), np.float32)
    rc = lib().orc_coo_to_csr(_p(keys), _p(vals), nnz, n_rows, n_cols, _p(rp), _p(ci), _p(ov))
    if rc == -1:
        raise ValueError("key outside [0, num_rows) x [0, num_cols)")
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    return rp, ci[:nnz], ov[:nnz]


def spmv(A: Csr, x: np.ndarray, threads: int = 1) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty(A.n, np.float64)
    if A.block == 0:
        lib().orc_csr_spmv(_p(A.row_ptr), _p(A.col_ind), _p(A.val), A.n, _p(x), _p(y), threads)
    else:
        lib().orc_bcsr_spmv(_p(A.row_ptr), _p(A.col_ind), _p(A.val), A.n // A.block,
                            A.block, _p(x), _p(y))
    return y


def _solve(name, A: Csr, b, compat, tol, max_iter, omega, threads, precond):
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(A.n, np.float64)
    o = _Opts(int(compat), int(max_iter), float(tol), float(omega), int(threads),
              {None: 0, "none": 0, "jacobi": 1}[precond])
    info = _Info()
    op = A._op()
    getattr(lib(), name)(C.byref(op), _p(b), _p(x), C.byref(o), C.byref(info))
    return x, {"iters": info.iters, "converged": bool(info.converged),
               "breakdown": bool(info.breakdown), "rel_resid": info.rel_resid}


def cg(A, b, compat=False, tol=1e-6, max_iter=2000, threads=1, precond=None):
    return _solve("orc_cg", A, b, compat, tol, max_iter, 0.0, threads, precond)


def bicgstab(A, b, compat=False, tol=1e-6, max_iter=2000, threads=1):
    return _solve("orc_bicgstab", A, b, compat, tol, max_iter, 0.0, threads, None)


def richardson(A, b, compat=True, omega=0.01, iters=1000, threads=1):
    return _solve("orc_richardson", A, b, compat, 0.0, iters, omega, threads, None)


def true_residual(A: Csr, b, x) -> float:
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    op = A._op()
    return float(lib().orc_true_residual(C.byref(op), _p(b), _p(x)))


# ---- learned FSAI (no reference counterpart) ------------------------------
NPARAM = 16 * 64 + 64 + 64 * 64 + 64 + 64 + 1


def fsai_pattern(A: Csr):
    """G's pattern (tril(A)): (row_ptr, col_ind, row, a_index)."""
    nnz = int(A.row_ptr[-1])
    rp = np.empty(A.n + 1, np.int32)
    ci = np.empty(max(nnz, 1), np.int32)
    row = np.empty(max(nnz, 1), np.int32)
    aidx = np.empty(max(nnz, 1), np.int32)
    op = A._op()
    k = lib().orc_fsai_pattern(C.byref(op), _p(rp), _p(ci), _p(row), _p(aidx))
    return rp, ci[:k], row[:k], aidx[:k]


def fsai_features(A: Csr):
    rp, ci, row, aidx = fsai_pattern(A)
    X = np.empty((ci.shape[0], 16), np.float32)
    op = A._op()
    lib().orc_fsai_features(C.byref(op), ci.shape[0], _p(row), _p(ci), _p(aidx), _p(X))
    return X, rp, ci, row


def mlp_forward(params, X):
    params = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    out = np.empty(X.shape[0], np.float64)
    lib().orc_mlp_forward(_p(params), _p(X), X.shape[0], _p(out))
    return out


def mlp_backward(params, X, dout):
    params = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    dout = np.ascontiguousarray(dout, dtype=np.float64)
    g = np.empty(NPARAM, np.float64)
    lib().orc_mlp_backward(_p(params), _p(X), X.shape[0], _p(dout), _p(g))
    return g


def fsai_value_map(out, row, col, diag):
    """g_ii = softplus(o + log(e-1)) / sqrt(a_ii), g_ij = o / sqrt(a_jj)."""
    out = np.asarray(out, np.float64)
    s = 1.0 / np.sqrt(diag[col])
    z = out + np.log(np.e - 1.0)
    sp = np.where(z > 20, z, np.log1p(np.exp(np.minimum(z, 20))))
    return np.where(row == col, sp * s, out * s)


def fsai_probe_loss_grad(A: Csr, G: Csr, V):
    V = np.ascontiguousarray(V, dtype=np.float64)
    k = V.shape[0]
    grad = np.empty(int(G.row_ptr[-1]), np.float64)
    opA, opG = A._op(), G._op()
    loss = lib().orc_fsai_probe_loss_grad(C.byref(opA), C.byref(opG), _p(V), k, _p(grad))
    return float(loss), grad
