"""B200-native (sm_100a) sparse iterative-solver path, drop-in for the
SparseForge/mpsparse PyTorch extensions.

    from mpsparse_b200 import spmv, bcsr, coo_csr
    A = spmv.csr_tensor(keys, values, row_ptr, col_ind, out_vals, n_rows, n_cols)
    A.cgd(b, x)            # x written in place

The native extension (``_C``) must have been built (``python -m
mpsparse_b200/build.py``); there is no CPU fallback, so importing the package
without it raises ImportError.
"""
from __future__ import annotations

import os as _os

_HERE = _os.path.dirname(_os.path.abspath(__file__))
LIB_PATH = _os.path.join(_HERE, "lib", "libmpsparse_b200.so")

try:
    import torch as _torch  # noqa: F401  (loads libtorch / libc10 for _C)
    from . import _C  # type: ignore[attr-defined]
except ImportError as _e:  # pragma: no cover - exercised only without a build
    raise ImportError(
        "mpsparse_b200's CUDA extension is not built or failed to load "
        f"({_e}); run `python mpsparse_b200/build.py` first"
    ) from _e

from . import spmv, bcsr, coo_csr  # noqa: E402,F401

__all__ = ["spmv", "bcsr", "coo_csr", "LIB_PATH"]
