"""Launch-shape autotuner: the coordinate-descent search on synthetic cost
functions and the C-ABI's host-side shape checks (CPU), then labels under
several shapes and a tuned BatchedPlan against the built-in shape (GPU)."""

import ctypes
import os

import numpy as np
import pytest
import torch

from dbscan_torch import tune

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "dbscan-torch_b200", "dbscan_torch", "libdbscan_b200.so")


class _Shape(ctypes.Structure):
    _fields_ = [("blocks_per_sm", ctypes.c_int32 * 6)]


def _cost(best):
    """Separable cost with its minimum at `best` (log distance per entry)."""
    def f(shape):
        return 10.0 + sum(abs(np.log2(v) - np.log2(b)) for v, b in zip(shape, best))
    return f


def test_descent_finds_separable_minimum():
    target = (16, 4, 32, 2, 8, 16)
    calls = []

    def measure(s):
        calls.append(s)
        return _cost(target)(s)

    shape, t, trials = tune.coordinate_descent(measure, (8,) * 6)
    assert shape == target and t == pytest.approx(10.0)
    assert len(calls) == len(set(calls)) == len(trials)  # each shape measured once
    assert len(trials) <= 1 + 6 * (len(tune.CANDIDATES) - 1)


def test_descent_ignores_gains_below_margin():
    # Every other shape is 0.5 % faster than the start: within the margin.
    shape, t, _ = tune.coordinate_descent(lambda s: 100.0 if s == (8,) * 6 else 99.5, (8,) * 6)
    assert shape == (8,) * 6 and t == 100.0


def test_descent_rejects_bad_shapes():
    with pytest.raises(ValueError):
        tune.coordinate_descent(lambda s: 1.0, (8,) * 5)
    with pytest.raises(ValueError):
        tune.coordinate_descent(lambda s: 1.0, (8,) * 6, candidates=(0, 8))
    with pytest.raises(ValueError):
        tune.coordinate_descent(lambda s: 1.0, (8,) * 5 + (64,))


def test_capi_shape_checks():
    """Host-side checks only: no CUDA call is reached."""
    lib = ctypes.CDLL(LIB)
    sh = _Shape()
    lib.dbs_default_launch_shape.argtypes = [ctypes.c_int64, ctypes.c_void_p]
    assert lib.dbs_default_launch_shape(10_000_000, ctypes.byref(sh)) == 0
    assert list(sh.blocks_per_sm) == [6, 8, 8, 8, 8, 32]
    assert lib.dbs_default_launch_shape((16 << 20) + 1, ctypes.byref(sh)) == 0
    assert list(sh.blocks_per_sm) == [6, 8, 8, 8, 8, 8]
    assert lib.dbs_default_launch_shape(10, None) == 1
    assert lib.dbs_default_launch_shape(-1, ctypes.byref(sh)) == 1
    f = lib.dbs_dbscan2d_batched_device_shaped
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    fake = ctypes.c_void_p(256)
    for bad in (-1, 33):
        b = _Shape()
        b.blocks_per_sm[3] = bad
        assert f(None, 0, 1, fake, fake, None, fake, 1 << 40, ctypes.byref(b), None) == 1
    ok = _Shape()
    ok.blocks_per_sm[0] = 32
    # n_total == 0: validated, then a no-op.
    assert f(None, 0, 1, fake, fake, None, fake, 1 << 40, ctypes.byref(ok), None) == 0
    assert f(None, 0, 1, fake, fake, None, fake, 1 << 40, None, None) == 0


def test_plan_set_shape_checks():
    """BatchedPlan.set_shape validates on the host and drops a captured graph
    (no device buffers needed: the plan object is built without __init__)."""
    from dbscan_torch import BatchedPlan
    plan = object.__new__(BatchedPlan)
    plan.graph = object()
    plan.set_shape([2, 4, 8, 16, 32, 0])
    assert plan.shape == (2, 4, 8, 16, 32, 0) and plan.graph is None
    for bad in [(8,) * 5, (8,) * 7, (33,) + (8,) * 5, (-1,) + (8,) * 5]:
        with pytest.raises(ValueError):
            plan.set_shape(bad)
    plan.set_shape(None)
    assert plan.shape is None


def _batch():
    from dbscan_torch import synthetic
    rng = np.random.default_rng(21)
    sizes = rng.integers(1, 40_000, size=40)
    sizes[[5, 11]] = 0
    clouds = [synthetic.blobs_with_noise(int(s), seed=300 + k, n_blobs=4) if s else
              np.zeros((0, 2), np.float32) for k, s in enumerate(sizes)]
    clouds.append(synthetic.constant_density(400_000, seed=3))
    eps = rng.uniform(0.3, 1.2, size=len(clouds))
    ms = rng.integers(2, 16, size=len(clouds))
    off = np.concatenate([[0], np.cumsum([len(c) for c in clouds])])
    return clouds, np.concatenate(clouds).astype(np.float32), off, eps, ms


SHAPES = [None, (1,) * 6, (32,) * 6, (2, 16, 1, 32, 4, 3), (0, 0, 5, 0, 7, 0)]


@pytest.mark.gpu
def test_labels_do_not_depend_on_shape():
    import oracle
    from dbscan_torch import BatchedPlan
    clouds, X, off, eps, ms = _batch()
    plan = BatchedPlan(off.tolist(), use_graph=False)
    Xd = torch.from_numpy(X).cuda()
    plan.set_params(eps, ms)
    outs = []
    for shape in SHAPES:
        plan.set_shape(shape)
        outs.append(plan.run(Xd).cpu().numpy().copy())
        assert plan.status() == 0
    for k, o in enumerate(outs[1:], 1):
        assert np.array_equal(o, outs[0]), f"shape {SHAPES[k]}"
    for k in (0, 7, len(clouds) - 1):
        want = oracle.dbscan2d(clouds[k], float(eps[k]), int(ms[k]))
        assert np.array_equal(outs[0][off[k]:off[k + 1]], want), f"cloud {k}"


@pytest.mark.gpu
def test_tuned_plan_replays_same_labels():
    from dbscan_torch import BatchedPlan, _C, dbscan2d_batched
    clouds, X, off, eps, ms = _batch()
    Xd = torch.from_numpy(X).cuda()
    want = dbscan2d_batched(Xd, off.tolist(), eps.tolist(), ms.tolist()).cpu().numpy()
    plan = BatchedPlan(off.tolist())
    plan.run(Xd, eps, ms)
    res = plan.tune(reps=2, candidates=(4, 8, 16))
    default = tuple(_C.default_launch_shape(int(off[-1])))
    assert res["default_shape"] == default and res["ms"] <= res["default_ms"]
    # Each entry is a candidate or the built-in value it started from.
    assert len(res["shape"]) == 6 and all(v in (4, 8, 16) or v == d for v, d in zip(res["shape"], default))
    assert plan.shape == res["shape"]
    for _ in range(2):  # capture with the tuned shape, then replay
        assert np.array_equal(plan.run(Xd).cpu().numpy(), want)
    assert plan.status() == 0
