"""Loader for the reference extension built by oracle/build_ref.py.

TEST INFRASTRUCTURE ONLY (tests/, the smoke check and the bench's reference
and CPU-baseline legs). Returns the reference's own pybind module `_C`
(csrc/extension.cpp:65-81 of ryanirl/dbscan-torch v0.2.0) or None when it was
not built.
"""

from __future__ import annotations

import glob
import importlib.machinery
import importlib.util
import os

HERE = os.path.dirname(os.path.abspath(__file__))
_cache: dict = {}


def load(kind: str = "cpu"):
    """kind: "cpu" (CPU-only build) or "cuda" (CPU + CUDA build)."""
    if kind in _cache:
        return _cache[kind]
    mod = None
    paths = sorted(glob.glob(os.path.join(HERE, "_ref", kind, "_C*.so")))
    if paths:
        import torch  # noqa: F401  (the module links against libtorch)
        loader = importlib.machinery.ExtensionFileLoader("_C", paths[0])
        spec = importlib.util.spec_from_file_location("_C", paths[0], loader=loader)
        mod = importlib.util.module_from_spec(spec)
        loader.exec_module(mod)
    _cache[kind] = mod
    return mod
