"""Generate the golden fixtures in this folder (committed .npz files).

The reference ships no golden vectors and runs only on Metal, so the fixtures
are built from the checks the reference itself treats as ground truth:

* COO -> CSR: ``torch.sparse_coo_tensor(...).to_sparse_csr()`` on unique keys
  (spmv_kernel/coo_csr/coo_csr/coo_csr/benchmark.py:133-156) and, for
  duplicate keys, a stable numpy argsort of the packed keys;
* SpMV: torch CSR matmul in float64 (spmv_kernel/spmv/benchmark.py:172-177);
* solver iterates: scipy.sparse.linalg.cg / bicgstab (the CPU solvers the
  reference benchmarks against, iterative/richardson/benchmark.py:169), first
  20 iterates from x0 = 0;
* Richardson: a float64 loop of iterative_op (iterative/richardson/spmv.cpp:
  376-425), 1000 iterations at w = 0.01.

Run: ``python tests/golden/make_golden.py`` (writes golden_*.npz here).
"""
from __future__ import annotations

import os
import sys

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mpsparse_b200 import workloads as W  # noqa: E402  (numpy generators only)

N_ITERATES = 20


def csr_by_torch(rows, cols, vals, n_rows, n_cols):
    coo = torch.sparse_coo_tensor(torch.stack([torch.from_numpy(rows), torch.from_numpy(cols)]),
                                  torch.from_numpy(vals), (n_rows, n_cols))
    csr = coo.to_sparse_csr()
    return (csr.crow_indices().numpy().astype(np.int32), csr.col_indices().numpy().astype(np.int32),
            csr.values().numpy().astype(np.float32))


def csr_stable(keys, vals, n_rows):
    order = np.argsort(keys.view(np.uint64), kind="stable")
    k = keys.view(np.uint64)[order]
    rows = (k >> np.uint64(32)).astype(np.int64)
    rp = np.zeros(n_rows + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    return (np.cumsum(rp).astype(np.int32), (k & np.uint64(0xFFFFFFFF)).astype(np.int32),
            vals[order].astype(np.float32))


def iterates(solver, A, b, n):
    xs = []
    solver(A, b, x0=np.zeros_like(b), rtol=1e-30, atol=0.0, maxiter=n,
           callback=lambda xk: xs.append(np.array(xk, dtype=np.float64)))
    return np.stack(xs[:n])


def main():
    rng = np.random.default_rng(1234)

    # 1. 12x12 Laplacian, shuffled (unique keys): CSR via torch, SpMV, CG.
    c = W.laplacian_2d(12).shuffled(7)
    keys = c.keys()
    rp, ci, cv = csr_by_torch(c.rows, c.cols, c.vals, c.n, c.n)
    A = sp.csr_matrix((cv.astype(np.float64), ci, rp), shape=(c.n, c.n))
    x = rng.standard_normal(c.n).astype(np.float32)
    y = torch.sparse_csr_tensor(torch.from_numpy(rp.astype(np.int64)),
                                torch.from_numpy(ci.astype(np.int64)),
                                torch.from_numpy(cv.astype(np.float64)), (c.n, c.n)) @ \
        torch.from_numpy(x.astype(np.float64))
    b = W.rhs(c.n, 11)
    cg_it = iterates(spla.cg, A, b.astype(np.float64), N_ITERATES)
    xr = np.zeros(c.n)
    for _ in range(1000):
        xr = xr + (0.01 * b - 0.01 * (A @ xr))
    np.savez_compressed(os.path.join(HERE, "golden_laplacian12.npz"), keys=keys, vals=c.vals,
                        n=c.n, row_ptr=rp, col_ind=ci, csr_vals=cv, x=x, y=y.numpy(), b=b,
                        cg_iterates=cg_it, richardson_x=xr)

    # 2. Random COO with duplicates, empty rows, non-square (stable order).
    n_rows, n_cols, nnz = 300, 77, 2000
    rows = rng.integers(0, n_rows // 2, nnz) * 2          # odd rows stay empty
    cols = rng.integers(0, n_cols, nnz)
    rows[:50] = rows[50:100]
    cols[:50] = cols[50:100]                                # duplicate keys
    keys = (rows.astype(np.int64) << 32) | cols.astype(np.int64)
    vals = rng.standard_normal(nnz).astype(np.float32)
    rp, ci, cv = csr_stable(keys, vals, n_rows)
    np.savez_compressed(os.path.join(HERE, "golden_duplicates.npz"), keys=keys, vals=vals,
                        n_rows=n_rows, n_cols=n_cols, row_ptr=rp, col_ind=ci, csr_vals=cv)

    # 3. Nonsymmetric diagonally dominant 4x4-block matrix: BCSR SpMV, BiCGSTAB.
    bm = W.block_dominant(16, 3, seed=5)
    coo = bm.to_coo(drop_zeros=False)
    Ab = sp.csr_matrix((coo.vals.astype(np.float64), (coo.rows, coo.cols)), shape=(bm.n, bm.n))
    xb = rng.standard_normal(bm.n).astype(np.float32)
    yb = Ab @ xb.astype(np.float64)
    bb = W.rhs(bm.n, 12)
    bicg_it = iterates(spla.bicgstab, Ab, bb.astype(np.float64), 8)
    np.savez_compressed(os.path.join(HERE, "golden_block16.npz"), row_ptr=bm.row_ptr,
                        col_ind=bm.col_ind, vals=bm.vals, n=bm.n, x=xb, y=yb, b=bb,
                        bicgstab_iterates=bicg_it)
    print("wrote golden_laplacian12.npz, golden_duplicates.npz, golden_block16.npz")


if __name__ == "__main__":
    main()
