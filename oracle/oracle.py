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
