"""Build the native parts of dbscan_torch in-tree.

  1. libdbscan_b200.so  -- the CUDA kernels and the C-ABI (include/dbscan_b200.h),
                          nvcc for sm_100a only, no torch dependency.
  2. _C*.so             -- the pybind11 torch extension (csrc/extension.cpp),
                          linked against libdbscan_b200.so with an $ORIGIN rpath.

Both land in dbscan_torch/ next to __init__.py so the package imports them
from the source tree (nothing is installed into site-packages).

Usage: python dbscan-torch_b200/build.py [--force] [-j N]
"""

from __future__ import annotations

import argparse
import ctypes
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
PKG = os.path.join(HERE, "dbscan_torch")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(PKG, "libdbscan_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

# sm_100a only. -ftz=true: single-precision subnormals flush to zero in every
# operation, as in the reference build's --use_fast_math device arithmetic.
# -fmad=false: no implicit multiply-add contraction; the kernels spell out
# the one fused multiply-add of the distance test themselves.
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-ftz=true", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "-I", INCLUDE,
]

CU_SOURCES = ["dbs_sort.cu", "dbs_csort.cu", "dbs_cells.cu", "dbs_cluster.cu", "dbs_capi.cu"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(force: bool = False, jobs: int = 4, verbose: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    objs = []
    procs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s] + headers):
            cmd = [NVCC, *NVCC_FLAGS, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((src, subprocess.Popen(cmd)))
            while len([p for _, p in procs if p.poll() is None]) >= jobs:
                procs[0][1].wait()
    for src, p in procs:
        if p.wait() != 0:
            raise RuntimeError(f"nvcc failed on {src}")
    if force or _newer(LIB, objs):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB, *objs,
               "-Xlinker", "--no-undefined", "-Xlinker", "-soname=libdbscan_b200.so"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def build_ext(force: bool = False, verbose: bool = True) -> str:
    import torch  # noqa: F401
    from torch.utils import cpp_extension

    src = os.path.join(CSRC, "extension.cpp")
    existing = glob.glob(os.path.join(PKG, "_C*.so"))
    deps = [src, os.path.join(INCLUDE, "dbscan_b200.h"), LIB]
    if existing and not force and not _newer(existing[0], deps):
        if not os.path.exists(os.path.join(PKG, "_build_info.py")):
            write_build_info()
        return existing[0]
    tmp = os.path.join(BUILD, "ext")
    os.makedirs(tmp, exist_ok=True)
    # The module's $ORIGIN rpath points at dbscan_torch/, not at the build
    # directory torch imports it from after linking: preload the library.
    ctypes.CDLL(LIB, mode=ctypes.RTLD_GLOBAL)
    cpp_extension.load(
        name="_C",
        sources=[src],
        extra_cflags=["-O3", "-std=c++17"],
        extra_include_paths=[INCLUDE],
        extra_ldflags=[f"-L{PKG}", "-ldbscan_b200", "-Wl,-rpath,\\$$ORIGIN"],
        build_directory=tmp,
        with_cuda=True,
        verbose=verbose,
    )
    built = glob.glob(os.path.join(tmp, "_C*.so"))
    if not built:
        raise RuntimeError("torch extension build produced no _C*.so")
    for old in existing:
        os.remove(old)
    dst = os.path.join(PKG, "_C.so")
    shutil.copy2(built[0], dst)
    write_build_info()
    return dst


def write_build_info() -> str:
    """Stamps the torch version the extension was built against into
    dbscan_torch/_build_info.py; the package refuses to import against another
    torch minor version (the extension's C++ ABI is tied to it)."""
    import torch
    path = os.path.join(PKG, "_build_info.py")
    with open(path, "w") as f:
        f.write('"""Written by build.py: the torch version the native extension was built against."""\n')
        f.write(f"BUILD_TORCH_VERSION = {torch.__version__!r}\n")
    return path


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=4)
    ap.add_argument("--lib-only", action="store_true")
    a = ap.parse_args(argv)
    print("lib ->", build_lib(a.force, a.j))
    if not a.lib_only:
        # The extension is built in a child process: torch's loader imports
        # the module it builds, and `_C` must not clash with other modules.
        r = subprocess.run([sys.executable, "-c",
                            f"import sys; sys.path.insert(0, {HERE!r}); import build; "
                            f"print('ext ->', build.build_ext({a.force!r}, False))"])
        if r.returncode != 0:
            return r.returncode
    return 0


if __name__ == "__main__":
    sys.exit(main())
