"""ctypes binding of include/mpsparse.h used by the tests to call the C ABI
directly (device pointers come from torch CUDA tensors)."""
import ctypes as C
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "mpsparse_b200", "lib", "libmpsparse_b200.so")
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
           if f.endswith(".h")]


class SolveOpts(C.Structure):
    _fields_ = [("reference_compat", C.c_int32), ("max_iter", C.c_int32), ("tol", C.c_double),
                ("omega", C.c_double), ("precond", C.c_int32), ("stall_window", C.c_int32),
                ("host_loop", C.c_int32), ("reserved", C.c_int32)]


class SolveInfo(C.Structure):
    _fields_ = [("iters", C.c_int32), ("converged", C.c_int32), ("breakdown", C.c_int32),
                ("stalled", C.c_int32), ("compat_snapshot", C.c_int32), ("stop_rule_met", C.c_int32),
                ("rel_resid", C.c_double), ("true_resid", C.c_double), ("persistent", C.c_int32),
                ("reserved", C.c_int32)]


def declared_symbols():
    names = set()
    for h in HEADERS:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names.update(re.findall(r"\b(mps_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB)
        vp, u64, u32, i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int32
        L.mps_csr_create_from_keys.argtypes = [vp, vp, u64, u32, u32, C.POINTER(vp), vp]
        L.mps_csr_destroy.argtypes = [vp]
        L.mps_csr_spmv.argtypes = [vp, vp, vp, vp]
        L.mps_csr_spmv_dot.argtypes = [vp, vp, vp, vp, vp, vp]
        L.mps_csr_export.argtypes = [vp, vp, vp, vp, vp]
        L.mps_coo_to_csr.argtypes = [vp, vp, u64, u32, u32, vp, vp, vp, vp]
        for f in ("mps_csr_cg", "mps_csr_bicgstab", "mps_csr_richardson"):
            getattr(L, f).argtypes = [vp, vp, vp, C.POINTER(SolveOpts), C.POINTER(SolveInfo), vp]
        L.mps_solve_opts_default.argtypes = [C.POINTER(SolveOpts)]
        L.mps_solve_opts_default.restype = None
        L.mps_last_error_string.restype = C.c_char_p
        L.mps_status_string.restype = C.c_char_p
        L.mps_status_string.argtypes = [C.c_int]
        _lib = L
    return _lib


def ptr(t):
    return C.c_void_p(t.data_ptr())


def check(status):
    if status != 0:
        raise RuntimeError(f"status {status}: {lib().mps_last_error_string().decode()}")
