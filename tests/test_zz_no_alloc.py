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


def _dense_rows_coo():
    """Short rows plus a few long ones: a row of 1,500 nonzeros inside a
    staged tile (its tile averages more than 16 nonzeros per row: one warp
    per row) and rows of 10k and 25k nonzeros, longer than a tile's staging
    capacity (the whole CTA strides each)."""
    rng = np.random.default_rng(3)
    n = 30000
    lens = rng.integers(1, 9, n)
    lens[11] = 1500
    lens[15000] = 10000
    lens[20000] = 25000
    rows = np.repeat(np.arange(n, dtype=np.int64), lens)
    cols = np.concatenate([np.sort(rng.choice(n, l, replace=False)) for l in lens]).astype(np.int64)
    vals = rng.standard_normal(rows.shape[0]).astype(np.float32)
    return W.Coo(rows, cols, vals, n).shuffled(4)


CASES = {
    "diffusion_400x300": lambda: W.lognormal_diffusion_2d(400, 300, 1.0, 8.0, 5).shuffled(2),
    "dense_rows": _dense_rows_coo,
    # about 5M nonzeros: more tiles than one wave of CTAs holds
    "laplacian_1000x1000": lambda: W.laplacian_2d(1000).shuffled(6),
}


@pytest.mark.parametrize("case", list(CASES))
def test_noalloc_matches_regular_entry_point(mps, oracle, case):
    L, noalloc = _noalloc()
    coo = CASES[case]()
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
            # and against the CPU oracle in FP64 (FP32 accumulation bound)
            Ao = oracle.Csr(rp.cpu().numpy(), ci.cpu().numpy(), cv.cpu().numpy(), n)
            xh = x.cpu().numpy().astype(np.float64)
            yo = oracle.spmv(Ao, xh)
            bound = oracle.spmv(oracle.Csr(Ao.row_ptr, Ao.col_ind, np.abs(Ao.val), n), np.abs(xh))
            assert np.all(np.abs(y.cpu().numpy() - yo) <= 1e-6 * bound + 1e-30), call
            wh = w.cpu().numpy().astype(np.float64)
            dot_bound = np.abs(wh) @ bound
            assert abs(d.item() - wh @ yo) <= 1e-6 * dot_bound + 1e-30, call
    finally:
        L.mps_csr_destroy(h)


def test_noalloc_rejects_unaligned_arrays(mps):
    L, noalloc = _noalloc()
    buf = torch.zeros(64, device="cuda")
    ibuf = torch.zeros(64, dtype=torch.int32, device="cuda")
    rp = torch.tensor([0, 4, 8], dtype=torch.int32, device="cuda")
    off = C.c_void_p(buf.data_ptr() + 4)               # 4-byte offset: not 16-byte aligned
    st = noalloc(cabi.ptr(rp), cabi.ptr(ibuf), off, 2, 2, 8, cabi.ptr(buf), cabi.ptr(buf),
                 cabi.ptr(buf), cabi.ptr(buf), None)
    assert st == 1 and b"aligned" in L.mps_last_error_string()


def test_noalloc_rejects_matrices_above_limit(mps):
    L, noalloc = _noalloc()
    too_many = (1 << 25) + 1
    dummy = torch.zeros(4, device="cuda")
    st = noalloc(cabi.ptr(dummy), cabi.ptr(dummy), cabi.ptr(dummy), 4, 4, too_many,
                 cabi.ptr(dummy), cabi.ptr(dummy), cabi.ptr(dummy), cabi.ptr(dummy), None)
    assert st == 1
    assert b"limit" in L.mps_last_error_string()
