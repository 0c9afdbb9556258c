"""ctypes front end of the CPU restatement oracle (oracle/dbscan_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the bench's
CPU-baseline leg as the checker. The product never imports this module.

The oracle restates the label semantics of the reference's CUDA path
(csrc/cuda/dbscan_cuda.cu:531-750 of ryanirl/dbscan-torch v0.2.0), see the
header of dbscan_oracle.c for the stage-by-stage citations.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

FORM_UNFUSED, FORM_FMA_X, FORM_FMA_Y = 0, 1, 2
SITES = (
    "core_box",     # point_box_d2 in k_core_pass2       dbscan_cuda.cu:235
    "core_pair",    # ex*ex+ey*ey in k_core_pass2        dbscan_cuda.cu:239
    "unite_bb",     # box_box_d2 in k_unite_pairs        dbscan_cuda.cu:351
    "unite_box",    # point_box_d2 in k_unite_pairs      dbscan_cuda.cu:359
    "unite_pair",   # ex*ex+ey*ey in k_unite_pairs       dbscan_cuda.cu:363
    "border_box",   # point_box_d2 in k_border_assign    dbscan_cuda.cu:453
    "border_pair",  # ex*ex+ey*ey in k_border_assign     dbscan_cuda.cu:458
)

# Arithmetic form of each call site in the reference build (nvcc 12.9,
# --use_fast_math, sm_100), settled by black-box label tests on a B200
# (tests/test_ref_cuda_forms.py): every site computes fma(ex, ex, ey*ey).
REFERENCE_FORMS = (FORM_FMA_X,) * len(SITES)

_lib = None


def build() -> str:
    """Compile the oracle (make in oracle/); returns the library path."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        p = ctypes.c_void_p
        lib.oracle_dbscan2d.restype = ctypes.c_int64
        lib.oracle_dbscan2d.argtypes = [p, ctypes.c_int64, ctypes.c_double, ctypes.c_int32,
                                        p, p, p, p, p, p, p, p, p, p, p, p]
        lib.oracle_pair_d2.restype = ctypes.c_float
        lib.oracle_pair_d2.argtypes = [ctypes.c_float] * 4 + [ctypes.c_int32]
        lib.oracle_pair_d2_batch.restype = None
        lib.oracle_pair_d2_batch.argtypes = [p, p, ctypes.c_int64, ctypes.c_int32, p]
        _lib = lib
    return _lib


def _i32(v: int) -> int:
    """static_cast<int32_t> of an int64 (dbscan_cuda.cu:550)."""
    return ((int(v) + 2**31) % 2**32) - 2**31


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def dbscan2d(X, eps: float, min_samples: int, forms=None, debug: bool = False):
    """Labels (int32, input order) of the reference CUDA path's semantics.

    With ``debug=True`` returns a dict holding the 11 intermediates of
    ``dbscan2d_cuda_debug`` (dbscan_cuda.cu:777-789), trimmed to num_cells.
    """
    lib = _load()
    X = np.ascontiguousarray(np.asarray(X, dtype=np.float32).reshape(-1, 2))
    n = X.shape[0]
    labels = np.full(n, -1, dtype=np.int32)
    f = np.asarray(REFERENCE_FORMS if forms is None else forms, dtype=np.int32)
    assert f.shape == (len(SITES),)
    if n == 0:
        return labels if not debug else {"labels": labels, "num_cells": 0}
    dbg = None
    if debug:
        dbg = dict(
            keys_sorted=np.empty(n, np.uint64), perm=np.empty(n, np.int32),
            xs=np.empty(n, np.float32), ys=np.empty(n, np.float32),
            is_core=np.empty(n, np.uint8), cell_start=np.empty(n + 1, np.int32),
            cluster_id_per_cell=np.empty(n, np.int32), uf=np.empty(n, np.int32),
            sorted_labels_pre_border=np.empty(n, np.int32),
            sorted_labels_final=np.empty(n, np.int32),
        )
    g = (lambda k: _ptr(dbg[k])) if debug else (lambda k: None)
    c = lib.oracle_dbscan2d(
        _ptr(X), n, float(eps), _i32(min_samples), _ptr(f), _ptr(labels),
        g("keys_sorted"), g("perm"), g("xs"), g("ys"), g("is_core"), g("cell_start"),
        g("cluster_id_per_cell"), g("uf"), g("sorted_labels_pre_border"),
        g("sorted_labels_final"))
    if c < 0:
        raise MemoryError("oracle allocation failed")
    if not debug:
        return labels
    dbg["cell_start"] = dbg["cell_start"][: c + 1]
    dbg["cluster_id_per_cell"] = dbg["cluster_id_per_cell"][:c]
    dbg["uf"] = dbg["uf"][:c]
    dbg["labels"] = labels
    dbg["num_cells"] = int(c)
    return dbg


def pair_d2(a, b, form: int) -> np.float32:
    """Device-rule squared distance of the pair (a, b) in one form."""
    lib = _load()
    return np.float32(lib.oracle_pair_d2(float(np.float32(a[0])), float(np.float32(a[1])),
                                         float(np.float32(b[0])), float(np.float32(b[1])), int(form)))


def pair_d2_batch(a: np.ndarray, b: np.ndarray, form: int) -> np.ndarray:
    """Device-rule squared distances of pairs (a[k], b[k]), ex = b - a."""
    lib = _load()
    a = np.ascontiguousarray(a, dtype=np.float32).reshape(-1, 2)
    b = np.ascontiguousarray(b, dtype=np.float32).reshape(-1, 2)
    out = np.empty(a.shape[0], dtype=np.float32)
    lib.oracle_pair_d2_batch(_ptr(a), _ptr(b), a.shape[0], int(form), _ptr(out))
    return out
