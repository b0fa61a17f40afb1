"""Batched solve: many independent SPD systems in one persistent launch.

``BatchedSolver.from_coo(keys, values, row_off)`` builds the block-diagonal
CSR on the GPU (the same radix sort as ``spmv.csr_tensor``) and hands it to
the persistent batched PCG (``mps_batch_*`` in the C ABI): every group of
warps of a persistent CTA takes the next system from a largest-first queue
and runs PCG on it to convergence, so thousands of systems cost one launch.

``prepare`` chooses the preconditioner per class of systems (the learned FSAI
factor where trial solves of a sample of the class say it does less work than
Jacobi) and lets the autotuner pick the warps per system.  ``solve`` returns
the per-system convergence record: iterations, converged flag (the mask) and
relative residual.  No reference counterpart: the reference solves one
system per call.
"""
from __future__ import annotations

import numpy as np
import torch

from ._C import batch_solver, csr_tensor

NONE, JACOBI, FSAI, SKIP = 0, 1, 2, 3


class BatchedSolver:
    def __init__(self, row_ptr, col_ind, vals, row_off):
        self.row_off = np.asarray(row_off, np.int64)
        self.n = int(self.row_off[-1])
        self.n_systems = len(self.row_off) - 1
        rp_at = row_ptr[torch.from_numpy(self.row_off).to(row_ptr.device)].cpu().numpy()
        self.nnz = np.diff(rp_at.astype(np.int64))           # nonzeros per system
        self.rows = np.diff(self.row_off)
        self.csr = (row_ptr, col_ind, vals)                  # the stacked CSR (device)
        self.impl = batch_solver(row_ptr, col_ind, vals,
                                 torch.from_numpy(self.row_off.astype(np.int32)))
        self.kinds = np.full(self.n_systems, JACOBI, np.int8)
        self.has_fsai = False

    @classmethod
    def from_coo(cls, keys, vals, row_off):
        """keys = (row << 32) | col with global (block-diagonal) indices."""
        n = int(row_off[-1])
        e = torch.empty(0)
        A = csr_tensor(keys, vals, e, e, e, n, n, fill_outputs=False)
        rp, ci, v = A.csr()
        del A
        return cls(rp, ci, v, row_off)

    def set_precond(self, kinds):
        kinds = np.ascontiguousarray(kinds, np.int8)
        self.impl.set_precond(torch.from_numpy(kinds))
        self.kinds = kinds

    def attach_fsai(self, fsai):
        self.impl.attach_fsai(fsai.model)
        self.has_fsai = True

    def iteration_cost(self, kind):
        """Bytes one PCG iteration of each system streams (FP32 values,
        int32 indices): A once, plus G and G^T (tril(A), about half of A
        each) for FSAI; about ten vector passes."""
        a = 8.0 * self.nnz + 4.0 * self.rows
        g = 8.0 * (self.nnz + self.rows) / 2 + 4.0 * self.rows
        vec = 40.0 * self.rows
        return a + vec + (2 * g if kind == FSAI else 0)

    def choose_precond(self, b, classes, tol=1e-6, max_iter=20000, sample=32):
        """Per class: solve a sample with Jacobi and with FSAI, keep the one
        with the smaller iterations x bytes-per-iteration total."""
        assert self.has_fsai, "attach_fsai first"
        classes = np.asarray(classes)
        kinds = np.full(self.n_systems, JACOBI, np.int8)
        x = torch.zeros(self.n, device=b.device)
        info = {}
        for c in np.unique(classes):
            idx = np.nonzero(classes == c)[0]
            pick = idx[np.unique(np.linspace(0, len(idx) - 1, min(sample, len(idx))).astype(int))]
            work = {}
            for kind in (JACOBI, FSAI):
                trial = np.full(self.n_systems, SKIP, np.int8)
                trial[pick] = kind
                self.set_precond(trial)
                it, _, _ = self.impl.cg(b, x, tol=tol, max_iter=max_iter)
                it = it.cpu().numpy().astype(np.float64)
                work[kind] = float((it[pick] * self.iteration_cost(kind)[pick]).sum())
            best = FSAI if work[FSAI] < work[JACOBI] else JACOBI
            kinds[idx] = best
            info[int(c)] = {"jacobi_bytes": work[JACOBI], "fsai_bytes": work[FSAI],
                            "chosen": "fsai" if best == FSAI else "jacobi"}
        self.set_precond(kinds)
        return info

    def autotune(self, b, tol=1e-6, max_iter=20000):
        wps, ms = self.impl.autotune(b, tol, max_iter)
        return {"warps_per_system": int(wps), "systems_on_clusters": int(self.impl.uses_clusters),
                "candidates_ms": dict(zip((1, 2, 4, 8, 16, 32), (float(t) for t in ms)))}

    def solve(self, b, x, tol=1e-6, max_iter=20000):
        """x (CUDA float32, total_rows) is overwritten.  Returns (iters,
        converged, relres) per system, on the device; no host sync."""
        return self.impl.cg(b, x, tol=tol, max_iter=max_iter)

    def solve_mixed(self, b, x64, tol=1e-6, inner_tol=1e-3, max_iter=20000):
        """Mixed precision: x64 (CUDA float64, total_rows) receives every
        system's solution accumulated in FP64; each system's residual is
        replaced by its FP64 b - A x as it drops, and a system stops only when
        that true residual meets tol.  Returns (iters, converged, FP64 true
        relative residual) per system, on the device; no host sync."""
        return self.impl.cg_mixed(b, x64, tol=tol, inner_tol=inner_tol, max_iter=max_iter)

    @property
    def warps_per_system(self):
        return self.impl.warps_per_system
