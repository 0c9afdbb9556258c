"""Host-side behaviour that needs no GPU: argument validation with the
reference's error messages (extension.cpp:26-31, tested by the reference in
test_basic.py:67-75), empty input, and the C-ABI library itself -- it loads,
exports every symbol include/dbscan_b200.h declares, sizes workspaces and
rejects bad arguments before touching a device."""

import ctypes
import os
import re

import numpy as np
import pytest
import torch

from dbscan_torch import DBSCAN, _C, dbscan2d, dbscan2d_batched

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dbscan_b200.h")
LIB = os.path.join(ROOT, "dbscan-torch_b200", "dbscan_torch", "libdbscan_b200.so")


def test_input_validation():
    with pytest.raises(RuntimeError, match=r"shape \(N, 2\)"):
        dbscan2d(torch.zeros((10, 3)), eps=1.0, min_samples=5)
    with pytest.raises(RuntimeError, match="float32"):
        dbscan2d(torch.zeros((10, 2), dtype=torch.float64), eps=1.0, min_samples=5)
    with pytest.raises(RuntimeError, match="eps"):
        dbscan2d(torch.zeros((10, 2)), eps=0.0, min_samples=5)
    with pytest.raises(RuntimeError, match="min_samples"):
        dbscan2d(torch.zeros((10, 2)), eps=1.0, min_samples=0)
    with pytest.raises(RuntimeError, match=r"shape \(N, 2\)"):
        dbscan2d(torch.zeros((10,)), eps=1.0, min_samples=5)


def test_empty_cpu():
    labels = dbscan2d(torch.empty((0, 2), dtype=torch.float32), eps=1.0, min_samples=5)
    assert labels.shape == (0,) and labels.dtype == torch.int32


def test_profile_empty():
    lab, prof = _C.dbscan2d_profile(torch.empty((0, 2)), 1.0, 5)
    assert lab.shape == (0,)
    assert list(prof) == sorted(["cell_keys", "sort_gather", "boundary_scan", "build_ngh",
                                 "core_mark", "union_find", "cluster_id", "core_labels",
                                 "border_assign", "unpermute"])


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU error path")
def test_no_gpu_fails_loudly():
    with pytest.raises(RuntimeError, match="CUDA device"):
        dbscan2d(torch.zeros((10, 2)), eps=1.0, min_samples=5)
    with pytest.raises(RuntimeError, match="CUDA device"):
        DBSCAN(eps=1.0, min_samples=5).fit(np.zeros((10, 2), np.float32))


def test_batched_validation():
    X = torch.zeros((10, 2))
    with pytest.raises(RuntimeError, match="seg_offsets"):
        dbscan2d_batched(X, [0, 5], [0.5, 0.5], [5, 5])
    with pytest.raises(RuntimeError, match="eps"):
        dbscan2d_batched(X, [0, 5, 10], [0.5, 0.0], [5, 5])
    with pytest.raises(RuntimeError, match="min_samples"):
        dbscan2d_batched(X, [0, 5, 10], [0.5, 0.5], [5, 0])
    with pytest.raises(RuntimeError, match="non-decreasing"):
        dbscan2d_batched(X, [0, 6, 4, 10], [0.5] * 3, [5] * 3)


def _declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(dbs_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_symbols_exported():
    lib = ctypes.CDLL(LIB)
    names = _declared_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), f"{n} declared in dbscan_b200.h but not exported"


def test_capi_host_checks():
    lib = ctypes.CDLL(LIB)
    lib.dbs_workspace_bytes.restype = ctypes.c_size_t
    lib.dbs_workspace_bytes.argtypes = [ctypes.c_int64, ctypes.c_int32]
    ws1 = lib.dbs_workspace_bytes(1_000_000, 1)
    ws2 = lib.dbs_workspace_bytes(2_000_000, 1)
    assert 0 < ws1 < ws2
    assert lib.dbs_workspace_bytes(-1, 1) == 0
    assert lib.dbs_workspace_bytes(10, 0) == 0
    f = lib.dbs_dbscan2d
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int64, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    assert f(None, 10, 0.0, 5, None, None, 0, None) == 1      # DBS_ERR_INVALID (eps)
    assert f(None, 10, 1.0, 0, None, None, 0, None) == 1      # min_samples
    assert f(None, -1, 1.0, 5, None, None, 0, None) == 1      # n < 0
    assert f(None, 2**31, 1.0, 5, None, None, 0, None) == 3   # DBS_ERR_TOO_LARGE
    buf = ctypes.create_string_buffer(512)
    assert f(buf, 10, 1.0, 5, buf, None, 0, None) == 2        # no workspace
    assert f(None, 0, 1.0, 5, None, ctypes.c_void_p(256), 1 << 40, None) == 0  # n == 0: no-op
    lib.dbs_strerror.restype = ctypes.c_char_p
    assert lib.dbs_strerror(2) == b"workspace missing, misaligned or too small"
    lib.dbs_stage_name.restype = ctypes.c_char_p
    assert [lib.dbs_stage_name(i).decode() for i in range(10)][:2] == ["cell_keys", "sort_gather"]
    assert lib.dbs_stage_name(10) is None


def test_fill_seg_params_matches_reference_scalars():
    # dbscan_cuda.cu:547-550: host float arithmetic.
    p = _C.fill_seg_params(torch.tensor([0.5, 0.3, 1e-3], dtype=torch.float64),
                           torch.tensor([10, 4, 2**33 + 7]))
    rec = p.numpy().view(np.float32).reshape(3, 4)
    ms = p.numpy().view(np.int32).reshape(3, 4)[:, 2]
    for k, e in enumerate([0.5, 0.3, 1e-3]):
        fe = np.float32(e)
        assert rec[k, 0] == np.float32(np.sqrt(np.float32(2.0))) / fe
        assert rec[k, 1] == fe * fe
    assert ms.tolist() == [10, 4, 7]
