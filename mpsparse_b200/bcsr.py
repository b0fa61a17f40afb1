"""Module ``bcsr``: the block-CSR solver object, as the reference's ``bcsr``
extension exposes it (iterative/BiCGSTAB/bcsr.cpp:953-966).

``bcsr_tensor(keys, values, row_ptr, col_ind, num_rows, num_cols, block_size=4)``
takes pre-built BCSR arrays (row-major B x B blocks, as scipy's
``bsr.data.flatten()``), or -- when ``row_ptr`` is empty -- packed COO keys
with their values, from which the BCSR is built on the GPU.  ``cgd(b, x)`` and
``bicgstab(b, x)`` accept ``b`` padded to a multiple of B or unpadded.
"""
from ._C import bcsr_tensor  # noqa: F401

__all__ = ["bcsr_tensor"]
