"""Raw-label parity on every benchmark workload, at full size.

Each workload the bench times is checked here label for label (bit-exact:
cluster numbering, noise and the (d2, input index) border tie rule) against
the C oracle and, when it is present in oracle/_ref/cuda, against the
reference's own CUDA build run on the same device:

  blobs_100k             100,000 points, 20 blobs + 5% noise, eps 0.5, ms 10
  constant_density_*     1M, 5M and 10M points at constant density, eps 0.5, ms 10
  adversarial_4M_ms*     4M points: a 2M-point 0.2 x 0.2 square (a few huge
                         cells: the hot-key counting sort), 64 spirals (deep
                         union-find chains), a lattice at exactly eps; ms 4, 32
  batch_4096             the 4,096-cloud batch (151M points) in one batched
                         run: every cloud against the reference CUDA build, a
                         seeded sample of clouds over the whole size range and
                         eps < 0.35 (where the stencil's corner cells hold
                         within-eps pairs) against the oracle

The oracle restates the reference CUDA path (csrc/cuda/dbscan_cuda.cu of
ryanirl/dbscan-torch v0.2.0) and is pinned to golden vectors made by that
build (tests/test_oracle.py).
"""

import functools

import numpy as np
import pytest
import torch

import oracle
import refmod
from dbscan_torch import _C, dbscan2d_batched, synthetic

pytestmark = pytest.mark.gpu


@functools.lru_cache(maxsize=1)
def _cloud(kind: str, n: int) -> np.ndarray:
    if kind == "blobs":
        return synthetic.blobs_with_noise(n, seed=0)
    if kind == "constant_density":
        return synthetic.constant_density(n, seed=0)
    return synthetic.adversarial(n, seed=0)


# name, generator kind, points, eps, min_samples, sort form expected
# (1: counting sort over the dense key space; every workload here is dense)
WORKLOADS = [
    ("blobs_100k", "blobs", 100_000, 0.5, 10, 1),
    ("constant_density_1M", "constant_density", 1_000_000, 0.5, 10, 1),
    ("constant_density_5M", "constant_density", 5_000_000, 0.5, 10, 1),
    ("constant_density_10M", "constant_density", 10_000_000, 0.5, 10, 1),
    ("adversarial_4M_ms4", "adversarial", 4_000_000, 0.5, 4, 1),
    ("adversarial_4M_ms32", "adversarial", 4_000_000, 0.5, 32, 1),
]


def _first_diff(got, want):
    d = np.flatnonzero(got != want)
    return f"{d.size}/{got.size} labels differ, first at {d[:8].tolist()}"


@pytest.mark.parametrize("name,kind,n,eps,ms,form", WORKLOADS, ids=[w[0] for w in WORKLOADS])
def test_workload_labels(name, kind, n, eps, ms, form):
    X = _cloud(kind, n)
    Xd = torch.from_numpy(X).cuda()
    ours, info = _C.dbscan2d_info(Xd, eps, ms)
    assert info["passes"] == 0 and info["sort_form"] == form, info
    got = ours.cpu().numpy()
    want = oracle.dbscan2d(X, eps, ms)
    assert np.array_equal(got, want), f"{name} vs oracle: {_first_diff(got, want)}"
    ref = refmod.load("cuda")
    if ref is not None:
        rl = ref.dbscan2d(Xd, eps, ms).cpu().numpy()
        assert np.array_equal(got, rl), f"{name} vs reference CUDA: {_first_diff(got, rl)}"
    if kind == "adversarial":
        # The 2M-point square is one hot key at least: the count pass ranked
        # its rows through the hot-key table.
        assert info["hot_slots"] >= 1, info


def _batch_sample(sizes, eps, seed=0, n_spread=48, n_small_eps=24):
    """Cloud indices: n_spread clouds at evenly spaced size ranks (smallest
    and largest included), plus n_small_eps clouds with eps < 0.35 drawn with
    a seeded generator, half of them from the largest quarter."""
    order = np.argsort(sizes, kind="stable")
    pick = set(order[np.linspace(0, len(order) - 1, n_spread).round().astype(int)].tolist())
    rng = np.random.default_rng(seed)
    small = np.flatnonzero(eps < 0.35)
    big = small[sizes[small] >= np.quantile(sizes, 0.75)]
    pick |= set(rng.choice(big, size=min(n_small_eps // 2, big.size), replace=False).tolist())
    rest = np.setdiff1d(small, np.fromiter(pick, dtype=np.int64))
    pick |= set(rng.choice(rest, size=min(n_small_eps - n_small_eps // 2, rest.size), replace=False).tolist())
    return sorted(pick)


def test_batch_4096_clouds():
    sizes, eps, ms = synthetic.batch_layout(4096, seed=0)
    X, off = synthetic.blobs_with_noise_device(sizes, seed=0, device="cuda")
    offl = off.tolist()
    lab = dbscan2d_batched(X, offl, eps, ms)
    _C.check_status()
    sample = _batch_sample(sizes, eps)
    assert len(sample) >= 64
    assert sum(eps[k] < 0.35 for k in sample) >= 16
    assert min(sizes[k] for k in sample) == sizes.min() and max(sizes[k] for k in sample) == sizes.max()
    for k in sample:
        a, b = offl[k], offl[k + 1]
        got = lab[a:b].cpu().numpy()
        want = oracle.dbscan2d(X[a:b].cpu().numpy(), float(eps[k]), int(ms[k]))
        assert np.array_equal(got, want), f"cloud {k} (n={b - a}, eps={eps[k]:.3f}, ms={ms[k]}): " \
                                          f"{_first_diff(got, want)}"
    ref = refmod.load("cuda")
    if ref is None:
        return
    bad = []
    for k in range(len(sizes)):
        a, b = offl[k], offl[k + 1]
        want = ref.dbscan2d(X[a:b], float(eps[k]), int(ms[k]))
        if not torch.equal(lab[a:b], want):
            bad.append(k)
    assert not bad, f"{len(bad)} of {len(sizes)} clouds differ from the reference CUDA build: {bad[:10]}"
