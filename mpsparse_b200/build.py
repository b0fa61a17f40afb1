"""In-tree build of the native parts.

1. ``lib/libmpsparse_b200.so`` -- the C-ABI library (include/mpsparse.h):
   every ``csrc/*.cu`` compiled by nvcc for sm_100a only.
2. ``_C*.so`` -- the C++ torch extension (pybind11) that mirrors the
   reference's ``spmv`` / ``bcsr`` / ``coo_csr`` modules on top of the C ABI.

Rebuilds only what is older than its sources.  Run it as a script,
``python mpsparse_b200/build.py`` (importing the package needs the built
extension, so this file imports nothing from it).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libmpsparse_b200.so")
OBJDIR = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    return r


def build_lib(verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    hdrs = _headers()
    objs, todo = [], []
    for cu in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(OBJDIR, os.path.basename(cu) + ".o")
        objs.append(obj)
        if _newer(obj, [cu] + hdrs):
            todo.append([NVCC] + NVCC_FLAGS + ["-I", os.path.join(ROOT, "include"), "-c", cu, "-o", obj])
    # translation units compile independently: one nvcc per host core
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        for r in ex.map(_run, todo):
            if verbose:
                sys.stderr.write(r.stderr)
    if _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda"])
    return LIB


def build_ext(verbose: bool = False) -> str:
    import torch
    from torch.utils import cpp_extension as ce

    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    out = os.path.join(HERE, "_C" + suffix)
    src = os.path.join(CSRC, "torch_ext.cpp")
    if not _newer(out, [src, LIB] + _headers()):
        return out
    inc = ce.include_paths() + [sysconfig.get_paths()["include"], os.path.join(ROOT, "include"),
                                "/usr/local/cuda/include"]
    libdirs = ce.library_paths()
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cmd = ["g++", "-O2", "-fPIC", "-shared", "-std=c++17", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           "-DTORCH_EXTENSION_NAME=_C", "-DTORCH_API_INCLUDE_EXTENSION_H", src, "-o", out]
    cmd += [f"-I{p}" for p in inc]
    cmd += [f"-L{p}" for p in libdirs] + [f"-L{LIBDIR}"]
    cmd += ["-lmpsparse_b200", "-lc10", "-ltorch", "-ltorch_cpu", "-ltorch_python", "-lc10_cuda",
            "-ltorch_cuda", "-Wl,-rpath,$ORIGIN/lib"]
    cmd += [f"-Wl,-rpath,{p}" for p in libdirs]
    _run(cmd)
    return out


def build(verbose: bool = False):
    lib = build_lib(verbose)
    ext = build_ext(verbose)
    return lib, ext


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
