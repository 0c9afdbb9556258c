"""Build the reference dbscan-torch extension from its own sources into oracle/_ref/.

TEST INFRASTRUCTURE ONLY. The product never imports anything under oracle/.

The reference (ryanirl/dbscan-torch v0.2.0) ships three translation units:
  csrc/extension.cpp        pybind11 module `_C` (dispatch + input checks)
  csrc/cpu/dbscan_cpu.cpp   CPU wrapper around csrc/cpu/dbscan_grid.hpp
  csrc/cuda/dbscan_cuda.cu  the CUDA pipeline (the bit-exact label oracle)

They are compiled where they lie (nothing is copied into this repository) with
the reference's own flags (setup.py:70-83: `-O3 -std=c++17 -fopenmp` for C++,
`-O3 --use_fast_math -std=c++17` for nvcc, `-DWITH_CUDA`), for sm_100
(TORCH_CUDA_ARCH_LIST=10.0, the arch-list mechanism of setup.py:15-23).
OpenMP links against torch's bundled libgomp because this toolchain has no
libgomp.spec for `-fopenmp` at link time.

Outputs:
  oracle/_ref/cuda/_C*.so   CPU + CUDA reference (needs libtorch_cuda at import)
  oracle/_ref/cpu/_C*.so    CPU-only reference (fallback when the CUDA build fails)

Usage: python oracle/build_ref.py --src <reference checkout> [--cpu-only]
       (or set DBSCAN_REFERENCE_SRC instead of --src)
"""

from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SRC_ENV = "DBSCAN_REFERENCE_SRC"


def _build(name: str, sources: list[str], cuda: bool, out_dir: str) -> str:
    import torch
    from torch.utils import cpp_extension

    os.makedirs(out_dir, exist_ok=True)
    tmp = os.path.join(out_dir, "_tmp")
    os.makedirs(tmp, exist_ok=True)
    torch_lib = os.path.join(os.path.dirname(torch.__file__), "lib")
    cflags = ["-O3", "-std=c++17", "-fopenmp"]
    if cuda:
        cflags.append("-DWITH_CUDA")
    ldflags = [f"-L{torch_lib}", "-l:libgomp.so.1", f"-Wl,-rpath,{torch_lib}"]
    if cuda:
        os.environ["TORCH_CUDA_ARCH_LIST"] = "10.0"
    cpp_extension.load(
        name="_C",
        sources=sources,
        extra_cflags=cflags,
        extra_cuda_cflags=["-O3", "--use_fast_math", "-std=c++17"] if cuda else None,
        extra_ldflags=ldflags,
        build_directory=tmp,
        with_cuda=cuda,
        verbose=False,
    )
    built = glob.glob(os.path.join(tmp, "_C*.so"))
    if not built:
        raise RuntimeError(f"reference build {name} produced no _C*.so")
    dst = os.path.join(out_dir, os.path.basename(built[0]))
    shutil.copy2(built[0], dst)
    shutil.rmtree(tmp, ignore_errors=True)
    return dst


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=os.environ.get(SRC_ENV),
                    help=f"reference checkout (default: ${SRC_ENV})")
    ap.add_argument("--cpu-only", action="store_true")
    ap.add_argument("--one", choices=["cpu", "cuda"], help=argparse.SUPPRESS)
    args = ap.parse_args(argv)
    if not args.src:
        print(f"no reference checkout given (--src or ${SRC_ENV}); nothing built")
        return 0
    csrc = os.path.join(args.src, "csrc")
    if not os.path.isdir(csrc):
        print(f"reference sources not found at {csrc}; nothing built")
        return 0
    cpu_sources = [os.path.join(csrc, "extension.cpp"), os.path.join(csrc, "cpu", "dbscan_cpu.cpp")]
    if args.one == "cpu":
        print(" ->", _build("cpu", cpu_sources, False, os.path.join(OUT, "cpu")))
        return 0
    if args.one == "cuda":
        print(" ->", _build("cuda", cpu_sources + [os.path.join(csrc, "cuda", "dbscan_cuda.cu")],
                            True, os.path.join(OUT, "cuda")))
        return 0
    # One process per build: torch's loader renames a second `_C` in the same
    # process (PyInit__C_v1), and the module must keep its own name.
    kinds = ["cpu"] if args.cpu_only else ["cpu", "cuda"]
    rc = 0
    for kind in kinds:
        print(f"building reference {kind} path ...", flush=True)
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--src", args.src, "--one", kind])
        if r.returncode != 0:
            print(f"reference {kind} build failed (rc={r.returncode})", file=sys.stderr)
            rc = 1
    return rc


if __name__ == "__main__":
    sys.exit(main())
