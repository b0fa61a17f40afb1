"""The allocation-free SpMV + dot entry point (mps_csr_spmv_dot_noalloc).

It serves callers that cannot allocate device memory (a process whose HBM
budget is all handed to its own pool, or a path where an allocation's device
synchronisation is not allowed).  It must give the same result as the regular
entry point mps_csr_spmv_dot, on two calls in a row (the shared scratch is
reused and its counter must come back to zero), and reject matrices above its
stated limit.  This file is collected last so that a run stopping at the first
failure has run every other test before it."""
import ctypes as C

import numpy as np
import pytest
import torch

from mpsparse_b200 import workloads as W
from tests import cabi

pytestmark = pytest.mark.gpu


def _noalloc():
    L = cabi.lib()
    f = L.mps_csr_spmv_dot_noalloc
    vp = C.c_void_p
    f.argtypes = [vp, vp, vp, C.c_uint32, C.c_uint32, C.c_uint64, vp, vp, vp, vp, vp]
    f.restype = C.c_int
    return L, f


def test_noalloc_matches_regular_entry_point(mps):
    L, noalloc = _noalloc()
    coo = W.lognormal_diffusion_2d(400, 300, 1.0, 8.0, 5).shuffled(2)
    n, nnz = coo.n, coo.nnz
    keys = torch.from_numpy(coo.keys()).cuda()
    vals = torch.from_numpy(coo.vals).cuda()
    h = C.c_void_p()
    cabi.check(L.mps_csr_create_from_keys(cabi.ptr(keys), cabi.ptr(vals), nnz, n, n, C.byref(h), None))
    try:
        rp = torch.empty(n + 1, dtype=torch.int32, device="cuda")
        ci = torch.empty(nnz, dtype=torch.int32, device="cuda")
        cv = torch.empty(nnz, dtype=torch.float32, device="cuda")
        cabi.check(L.mps_csr_export(h, cabi.ptr(rp), cabi.ptr(ci), cabi.ptr(cv), None))
        g = torch.Generator(device="cuda").manual_seed(0)
        for call in range(2):                       # two calls in a row, new inputs each time
            x = torch.randn(n, device="cuda", generator=g)
            w = torch.randn(n, device="cuda", generator=g)
            y_ref = torch.empty(n, device="cuda")
            d_ref = torch.empty(1, dtype=torch.float64, device="cuda")
            cabi.check(L.mps_csr_spmv_dot(h, cabi.ptr(x), cabi.ptr(w), cabi.ptr(y_ref),
                                          cabi.ptr(d_ref), None))
            y = torch.full((n,), float("nan"), device="cuda")
            d = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
            cabi.check(noalloc(cabi.ptr(rp), cabi.ptr(ci), cabi.ptr(cv), n, n, nnz, cabi.ptr(x),
                               cabi.ptr(w), cabi.ptr(y), cabi.ptr(d), None))
            torch.cuda.synchronize()
            assert torch.allclose(y, y_ref, rtol=1e-6, atol=1e-6), call
            assert abs(d.item() - d_ref.item()) <= 1e-9 * abs(d_ref.item()) + 1e-9, call
    finally:
        L.mps_csr_destroy(h)


def test_noalloc_rejects_matrices_above_limit(mps):
    L, noalloc = _noalloc()
    too_many = (1 << 25) + 1
    dummy = torch.zeros(4, device="cuda")
    st = noalloc(cabi.ptr(dummy), cabi.ptr(dummy), cabi.ptr(dummy), 4, 4, too_many,
                 cabi.ptr(dummy), cabi.ptr(dummy), cabi.ptr(dummy), cabi.ptr(dummy), None)
    assert st == 1
    assert b"limit" in L.mps_last_error_string()
