"""The built-in scratch entry point, dbs_dbscan2d_static, called through the
C-ABI (ctypes on libdbscan_b200.so) and compared with the plain entry point
dbs_dbscan2d on the same inputs, two calls in a row.

The file name sorts last so that pytest collects it after every other test
file; it also passes alone in a fresh process (it loads the library itself).
"""

import ctypes
import os
import re

import numpy as np
import pytest
import torch

from dbscan_torch import synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dbscan_b200.h")
LIB = os.path.join(ROOT, "dbscan-torch_b200", "dbscan_torch", "libdbscan_b200.so")

DBS_OK = 0
DBS_ERR_INVALID = 1


def _define(name):
    m = re.search(rf"#define {name} \(?(\d+)u?(?: << (\d+)\))?", open(HEADER).read())
    assert m, name
    v = int(m.group(1))
    return v << int(m.group(2)) if m.group(2) else v


MAX_POINTS = _define("DBS_STATIC_MAX_POINTS")
SCRATCH_BYTES = _define("DBS_STATIC_SCRATCH_BYTES")
ERR_STATIC_LIMIT = _define("DBS_ERR_STATIC_LIMIT")


def _lib():
    lib = ctypes.CDLL(LIB)
    lib.dbs_workspace_bytes.restype = ctypes.c_size_t
    lib.dbs_workspace_bytes.argtypes = [ctypes.c_int64, ctypes.c_int32]
    lib.dbs_dbscan2d.restype = ctypes.c_int
    lib.dbs_dbscan2d.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int64,
                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    lib.dbs_dbscan2d_static.restype = ctypes.c_int
    lib.dbs_dbscan2d_static.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
                                        ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p]
    lib.dbs_strerror.restype = ctypes.c_char_p
    return lib


def test_static_limits():
    """Host-side checks only: no CUDA call is reached."""
    lib = _lib()
    assert MAX_POINTS == 16384 and SCRATCH_BYTES == 8 << 20
    # The largest accepted cloud fits the array with the workspace layout of
    # the plain entry point.
    assert 0 < lib.dbs_workspace_bytes(MAX_POINTS, 1) <= SCRATCH_BYTES
    f = lib.dbs_dbscan2d_static
    buf = ctypes.create_string_buffer(64)
    assert f(buf, MAX_POINTS + 1, 0.5, 5, buf, None, None) == ERR_STATIC_LIMIT
    assert f(buf, 1 << 40, 0.5, 5, buf, None, None) == ERR_STATIC_LIMIT
    assert b"DBS_STATIC_MAX_POINTS" in lib.dbs_strerror(ERR_STATIC_LIMIT)
    assert f(None, 10, 0.0, 5, None, None, None) == DBS_ERR_INVALID
    assert f(None, 10, 0.5, 0, None, None, None) == DBS_ERR_INVALID
    assert f(None, -1, 0.5, 5, None, None, None) == DBS_ERR_INVALID
    assert f(None, 10, 0.5, 5, None, None, None) == DBS_ERR_INVALID  # n > 0, no buffers
    assert f(None, 0, 0.5, 5, None, None, None) == DBS_OK


def _plain(lib, X, eps, ms, stream):
    n = X.shape[0]
    ws = torch.empty(lib.dbs_workspace_bytes(n, 1), dtype=torch.uint8, device=X.device)
    lab = torch.empty(n, dtype=torch.int32, device=X.device)
    rc = lib.dbs_dbscan2d(X.data_ptr(), n, eps, ms, lab.data_ptr(), ws.data_ptr(), ws.numel(), stream)
    assert rc == DBS_OK, lib.dbs_strerror(rc)
    torch.cuda.synchronize()
    return lab.cpu().numpy()


def _static(lib, X, eps, ms, stream):
    n = X.shape[0]
    lab = torch.full((n,), -7, dtype=torch.int32, device=X.device)
    st = torch.full((1,), 0xFFFF, dtype=torch.int32, device=X.device)
    rc = lib.dbs_dbscan2d_static(X.data_ptr(), n, eps, ms, lab.data_ptr(), st.data_ptr(), stream)
    assert rc == DBS_OK, lib.dbs_strerror(rc)
    torch.cuda.synchronize()
    assert st.item() == 0, f"device status {st.item():#x}"
    return lab.cpu().numpy()


@pytest.mark.gpu
def test_static_matches_plain_two_calls():
    lib = _lib()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # The largest accepted cloud, then a smaller one with other parameters, so
    # the second call runs on scratch the first one left behind.
    clouds = [(synthetic.blobs_with_noise(MAX_POINTS, seed=11, n_blobs=12), 1.0, 10),
              (synthetic.blobs_with_noise(3001, seed=12, n_blobs=5), 1.5, 4)]
    for Xn, eps, ms in clouds:
        X = torch.from_numpy(Xn).to(dev)
        want = _plain(lib, X, eps, ms, stream)
        got = _static(lib, X, eps, ms, stream)
        assert np.array_equal(got, want)
        assert len(set(want.tolist()) - {-1}) >= 2 and (want == -1).any()
    # n == 0 clears the status word.
    st = torch.full((1,), 5, dtype=torch.int32, device=dev)
    assert lib.dbs_dbscan2d_static(None, 0, 0.5, 5, None, st.data_ptr(), stream) == DBS_OK
    torch.cuda.synchronize()
    assert st.item() == 0
