"""Serving loop (dbscan_torch.serve): every request's labels equal the
oracle's labels for that cloud (bit-exact) and a plain dbscan2d call on that
cloud alone -- the same result alone and in the mix; admission respects the
lane capacity and the device-memory budget; queued requests are batched."""

import time

import numpy as np
import pytest
import torch

import oracle
from dbscan_torch import DbscanServer, dbscan2d, footprint_bytes, synthetic
from dbscan_torch import _C


def _check(r):
    """Request r's labels against the oracle and against a plain call alone."""
    want = oracle.dbscan2d(r.X.numpy(), r.eps, r.min_samples)
    got = r.labels.numpy()
    assert np.array_equal(got, want), f"request {r.rid} (n={r.n}): {(got != want).sum()} labels differ from the oracle"
    alone = dbscan2d(r.X.cuda(), r.eps, r.min_samples).cpu()
    assert torch.equal(r.labels, alone), f"request {r.rid} (n={r.n}): differs from the plain call"


def test_footprint_monotone():
    sizes = [0, 1, 1000, 100_000, 2_000_000]
    fp = [footprint_bytes(n) for n in sizes]
    assert all(a < b for a, b in zip(fp, fp[1:]))
    assert footprint_bytes(1000) >= _C.workspace_bytes(1000, 1) + 12 * 1000
    assert footprint_bytes(1000, 8) > footprint_bytes(1000, 1)


def _requests(k, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(k):
        n = int(np.exp(rng.uniform(np.log(1), np.log(60_000)))) if i % 11 else 0
        X = synthetic.blobs_with_noise(n, seed=seed * 1000 + i) if n else np.zeros((0, 2), np.float32)
        out.append((torch.from_numpy(X).pin_memory(), float(rng.uniform(0.1, 1.0)), int(rng.integers(4, 33))))
    return out


@pytest.mark.gpu
def test_serve_matches_plain():
    srv = DbscanServer(budget_bytes=2 << 30, lane_clouds=16)
    reqs = [srv.submit(X, e, m) for X, e, m in _requests(80, 1)]
    srv.drain()
    assert srv.completed == len(reqs) and srv.batches < len(reqs)
    for r in reqs:
        assert r.done and r.latency >= 0
        _check(r)


@pytest.mark.gpu
def test_serve_interleaved_submit():
    """Requests submitted while batches run (the loop is stepped between
    submissions): same labels as plain calls."""
    srv = DbscanServer(budget_bytes=1 << 30, lane_clouds=4, lanes=2)
    reqs = []
    for X, e, m in _requests(30, 2):
        reqs.append(srv.submit(X, e, m))
        srv.step()
    srv.drain()
    for r in reqs:
        _check(r)


@pytest.mark.gpu
def test_serve_admission():
    srv = DbscanServer(budget_bytes=256 << 20, lane_points=100_000, lane_clouds=8)
    assert srv.arena_bytes <= 256 << 20
    with pytest.raises(RuntimeError, match="exceeds the lane capacity"):
        srv.submit(torch.zeros((100_001, 2)), 0.5, 5)
    with pytest.raises(RuntimeError, match="eps"):
        srv.submit(torch.zeros((10, 2)), 0.0, 5)
    with pytest.raises(ValueError, match="budget"):
        DbscanServer(budget_bytes=64 << 20, lane_points=1_000_000)
    # A batch never exceeds the lane: 12 requests of 30k points -> batches of 3.
    X = torch.from_numpy(synthetic.blobs_with_noise(30_000, seed=5)).pin_memory()
    reqs = [srv.submit(X, 0.5, 10) for _ in range(12)]
    srv.drain()
    assert srv.batches >= 4
    want = torch.from_numpy(oracle.dbscan2d(X.numpy(), 0.5, 10))
    assert all(torch.equal(r.labels, want) for r in reqs)


@pytest.mark.gpu
def test_serve_pop_finished():
    """pop_finished() hands back every completed request exactly once, each
    with its labels, once a caller has asked for it."""
    srv = DbscanServer(budget_bytes=1 << 30, lane_clouds=4, lanes=3)
    assert srv.pop_finished() == []
    reqs = [srv.submit(X, e, m) for X, e, m in _requests(25, 3)]
    seen = []
    t_end = time.monotonic() + 120.0
    while len(seen) < len(reqs) and time.monotonic() < t_end:
        srv.step()
        seen.extend(srv.pop_finished())
    assert sorted(r.rid for r in seen) == sorted(r.rid for r in reqs)
    assert srv.pop_finished() == []
    for r in seen:
        assert r.done
        _check(r)


@pytest.mark.gpu
def test_pinned_arena_reuse():
    """The host arena hands out ranges first-fit, takes them back when the
    last view is released (coalescing neighbours) and counts the
    allocations it had to leave to torch's pinned allocator."""
    a = _C.PinnedArena(1 << 20)
    assert a.bytes == 1 << 20 and a.in_use == 0
    x = a.alloc_int32(1000)
    y = a.alloc_int32(50_000)
    assert x.is_pinned() and y.is_pinned() and a.in_use >= 204_000
    x.fill_(7)
    v = x[10:20]
    del x
    assert a.in_use >= 200_000  # the view keeps its range
    assert int(v.sum()) == 70
    del v, y
    assert a.in_use == 0
    big = a.alloc_int32(1 << 18)  # the whole arena: the freed ranges coalesced
    assert a.fallbacks == 0 and a.in_use == 1 << 20
    z = a.alloc_int32(10)  # nothing left: torch's pinned allocator
    assert a.fallbacks == 1 and z.is_pinned()
    del big, z
    assert a.in_use == 0
