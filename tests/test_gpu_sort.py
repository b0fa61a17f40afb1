"""COO -> CSR on the GPU: bit-exact against the oracle's stable sort."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _csr_gpu(mps, keys, vals, n_rows, n_cols):
    k = torch.from_numpy(np.ascontiguousarray(keys, dtype=np.int64)).cuda()
    v = torch.from_numpy(np.ascontiguousarray(vals, dtype=np.float32)).cuda()
    nnz = keys.shape[0]
    rp = torch.zeros(n_rows + 1, dtype=torch.int32)
    ci = torch.zeros(nnz, dtype=torch.int32)
    ov = torch.zeros(nnz, dtype=torch.float32)
    mps.coo_csr.coo_csr(k, v, rp, ci, ov, n_rows, n_cols)
    return rp.numpy(), ci.numpy(), ov.numpy()


def _assert_same(a, b):
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_golden_laplacian(mps, golden):
    g = golden("laplacian12")
    out = _csr_gpu(mps, g["keys"], g["vals"], int(g["n"]), int(g["n"]))
    _assert_same(out, (g["row_ptr"], g["col_ind"], g["csr_vals"]))


def test_golden_duplicates(mps, golden):
    g = golden("duplicates")
    out = _csr_gpu(mps, g["keys"], g["vals"], int(g["n_rows"]), int(g["n_cols"]))
    _assert_same(out, (g["row_ptr"], g["col_ind"], g["csr_vals"]))


@pytest.mark.parametrize("n_rows,n_cols,nnz,seed", [
    (1, 1, 1, 0), (1, 1, 5000, 1), (7, 3, 100, 2), (65536, 65536, 326656, 3),
    (1000, 2 ** 31 - 2, 300000, 4), (1 << 24, 1000, 300000, 5), (300000, 300000, 2_000_003, 6),
    (4096, 4096, 4096 * 8 + 17, 7)])
def test_random_vs_oracle(mps, oracle, n_rows, n_cols, nnz, seed):
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, n_rows, nnz)
    cols = rng.integers(0, n_cols, nnz)
    if nnz > 100:
        rows[: nnz // 10] = rows[nnz // 10: 2 * (nnz // 10)]   # duplicate keys
        cols[: nnz // 10] = cols[nnz // 10: 2 * (nnz // 10)]
    keys = (rows.astype(np.int64) << 32) | cols.astype(np.int64)
    vals = rng.standard_normal(nnz).astype(np.float32)
    if nnz <= 400000:
        ref = oracle.coo_to_csr(keys, vals, n_rows, n_cols)
    else:   # stable numpy sort (same definition; the oracle's 4-bit passes are slow here)
        order = np.argsort(keys, kind="stable")
        ref = (np.searchsorted(rows[order], np.arange(n_rows + 1)).astype(np.int32),
               cols[order].astype(np.int32), vals[order])
    _assert_same(_csr_gpu(mps, keys, vals, n_rows, n_cols), ref)


def test_shuffled_c1_matches_stable_sort(mps, oracle):
    from mpsparse_b200 import workloads as W
    c = W.laplacian_256().shuffled(0)
    ref = oracle.coo_to_csr(c.keys(), c.vals, c.n, c.n)
    _assert_same(_csr_gpu(mps, c.keys(), c.vals, c.n, c.n), ref)


def test_empty_and_out_of_range(mps):
    rp, ci, ov = _csr_gpu(mps, np.zeros(0, np.int64), np.zeros(0, np.float32), 5, 5)
    assert rp.tolist() == [0] * 6
    bad = np.array([(5 << 32) | 1], np.int64)
    with pytest.raises(RuntimeError, match="out of range"):
        _csr_gpu(mps, bad, np.ones(1, np.float32), 5, 5)
    bad = np.array([(1 << 32) | 9], np.int64)
    with pytest.raises(RuntimeError, match="out of range"):
        _csr_gpu(mps, bad, np.ones(1, np.float32), 5, 5)


def test_csr_tensor_fills_outputs_and_cabi(mps, golden):
    from tests import cabi
    g = golden("laplacian12")
    n = int(g["n"])
    keys = torch.from_numpy(g["keys"])
    vals = torch.from_numpy(g["vals"])
    rp = torch.zeros(n + 1, dtype=torch.int32)
    ci = torch.zeros(keys.numel(), dtype=torch.int32)
    ov = torch.zeros(keys.numel(), dtype=torch.float32)
    A = mps.spmv.csr_tensor(keys, vals, rp, ci, ov, n, n)
    assert np.array_equal(rp.numpy(), g["row_ptr"]) and np.array_equal(ci.numpy(), g["col_ind"])
    assert A.nnz == keys.numel()
    # the same through the raw C ABI
    import ctypes as C
    L = cabi.lib()
    h = C.c_void_p()
    kd, vd = keys.cuda(), vals.cuda()
    cabi.check(L.mps_csr_create_from_keys(cabi.ptr(kd), cabi.ptr(vd), keys.numel(), n, n,
                                          C.byref(h), None))
    r2 = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    c2 = torch.empty(keys.numel(), dtype=torch.int32, device="cuda")
    v2 = torch.empty(keys.numel(), dtype=torch.float32, device="cuda")
    cabi.check(L.mps_csr_export(h, cabi.ptr(r2), cabi.ptr(c2), cabi.ptr(v2), None))
    torch.cuda.synchronize()
    L.mps_csr_destroy(h)
    assert np.array_equal(r2.cpu().numpy(), g["row_ptr"])
    assert np.array_equal(v2.cpu().numpy(), g["csr_vals"])


def test_lookback_timeout_returns_error_and_device_stays_usable(mps, oracle):
    """A bounded device wait that runs out: the timeout hook makes tile 0
    publish no look-back status, so the later tiles' waits (bounded at 20,000
    polls, well under a second) give up.  The call returns MPS_ERR_TIMEOUT,
    and afterwards the device and the library still convert bit-exactly."""
    import ctypes as C
    from mpsparse_b200 import workloads as W
    from tests import cabi
    L = cabi.lib()
    f = L.mps_test_sort_lookback_timeout
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                  C.c_uint32, C.c_void_p]
    f.restype = C.c_int
    c = W.laplacian_2d(128).shuffled(3)               # 81,408 keys: 20 tiles
    keys = torch.from_numpy(c.keys()).cuda()
    vals = torch.from_numpy(c.vals).cuda()
    for _ in range(2):
        st = f(cabi.ptr(keys), cabi.ptr(vals), c.nnz, c.n, c.n, 20000, 0, None)
        assert st == 4, st                             # MPS_ERR_TIMEOUT
        assert b"bounded device wait" in L.mps_last_error_string()
    torch.cuda.synchronize()
    # the same hook with no silent tile is an ordinary conversion
    assert f(cabi.ptr(keys), cabi.ptr(vals), c.nnz, c.n, c.n, 20000, 0xFFFFFFFF, None) == 0
    out = _csr_gpu(mps, c.keys(), c.vals, c.n, c.n)
    _assert_same(out, oracle.coo_to_csr(c.keys(), c.vals, c.n, c.n))
