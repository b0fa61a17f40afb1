"""The C-ABI library loads and exports every declared entry point; host-side
argument checks work without a GPU."""
import ctypes as C

from tests import cabi


def test_exports_every_declared_symbol():
    L = cabi.lib()
    names = cabi.declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings_and_defaults():
    L = cabi.lib()
    assert L.mps_status_string(0) == b"ok"
    assert L.mps_status_string(6) == b"key out of range"
    o = cabi.SolveOpts()
    L.mps_solve_opts_default(C.byref(o))
    assert o.tol == 1e-6 and o.max_iter == 2000 and o.omega == 0.01 and o.host_loop == 0


def test_argument_checks_without_gpu():
    L = cabi.lib()
    h = C.c_void_p()
    # zero-sized shape and null outputs are rejected before any CUDA call
    assert L.mps_csr_create_from_keys(None, None, 0, 0, 4, C.byref(h), None) == 1
    assert b"positive" in L.mps_last_error_string()
    assert L.mps_csr_create_from_keys(None, None, 10, 4, 4, C.byref(h), None) == 1
    assert L.mps_csr_create_from_keys(None, None, 1 << 31, 4, 4, C.byref(h), None) == 1
    assert L.mps_csr_cg(None, None, None, None, None, None) == 1
    f = L.mps_test_sort_lookback_timeout
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                  C.c_uint32, C.c_void_p]
    assert f(None, None, 10, 4, 4, 100, 0, None) == 1
    assert L.mps_csr_destroy(None) == 0


def test_torch_extension_imports():
    import mpsparse_b200
    from mpsparse_b200 import spmv, bcsr, coo_csr
    assert mpsparse_b200._C.abi_version() == 4
    assert hasattr(spmv.csr_tensor, "cgd") and hasattr(spmv.csr_tensor, "bicgstab")
    assert hasattr(spmv.csr_tensor, "richardson") and hasattr(spmv.csr_tensor, "iter_solve")
    assert hasattr(bcsr.bcsr_tensor, "bicgstab") and callable(coo_csr.coo_csr)
