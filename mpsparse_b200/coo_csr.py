"""Module ``coo_csr``: the standalone converter
(spmv_kernel/coo_csr/coo_csr/coo_csr/coo_to_csr.cpp:259-288).

``coo_csr(keys, values, row_ptr, col_ind, out_vals, num_rows, num_cols)``
writes the CSR of the packed keys into the three caller tensors.
"""
from ._C import coo_csr  # noqa: F401

__all__ = ["coo_csr"]
