"""Module ``spmv``: the CSR solver object, as the reference's ``spmv``
extension exposes it (iterative/BiCGSTAB/spmv.cpp:892-905).

``csr_tensor(keys, values, row_ptr, col_ind, out_vals, num_rows, num_cols)``
sorts packed (row<<32|col) keys into CSR on the GPU.  Methods write their
output in place: ``mv(x, b)`` (b = A x), ``cgd(b, x)``, ``bicgstab(b, x)``,
``richardson(b, x)`` and ``iter_solve(b, x)`` (= cgd), plus ``cg_mixed`` (FP64
iterative refinement) and ``set_fsai`` (attach a learned factor G).
"""
from __future__ import annotations

import torch

from ._C import csr_tensor  # noqa: F401


def pack_keys(row_indices: torch.Tensor, col_indices: torch.Tensor) -> torch.Tensor:
    """(row << 32) | col as int64 (README.md:34-44 of the reference)."""
    return (row_indices.to(torch.int64) << 32) | col_indices.to(torch.int64)


__all__ = ["csr_tensor", "pack_keys"]
