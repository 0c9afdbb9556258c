"""Raw-label parity of the sm_100a pipeline with the oracle (and with the
reference's own CUDA build when it is present in oracle/_ref/cuda).

Bit-exact: labels are integers, so equality is exact -- cluster numbering,
noise and the (d2, perm[j]) border tie rule included. The debug entry point
is compared intermediate by intermediate (layout of dbscan_cuda.cu:777-789).
"""

import numpy as np
import pytest
import torch

import datasets
import oracle
import refmod
from dbscan_torch import _C, dbscan2d, dbscan2d_batched, synthetic

pytestmark = pytest.mark.gpu

CASES = datasets.parity_cases()
IDS = [c[0] for c in CASES]


@pytest.mark.parametrize("name,X,eps,ms", CASES, ids=IDS)
def test_labels_match_oracle(name, X, eps, ms):
    ours = dbscan2d(torch.from_numpy(X).cuda(), eps, ms).cpu().numpy()
    ref = oracle.dbscan2d(X, eps, ms)
    diff = np.flatnonzero(ours != ref)
    assert diff.size == 0, f"{name}: {diff.size}/{X.shape[0]} labels differ, first at {diff[:10]}"


@pytest.mark.parametrize("name,X,eps,ms", CASES[:12], ids=IDS[:12])
def test_debug_intermediates_match_oracle(name, X, eps, ms):
    out = _C.dbscan2d_cuda_debug(torch.from_numpy(X).cuda(), eps, ms)
    o = oracle.dbscan2d(X, eps, ms, debug=True)
    names = ["labels", "keys_sorted", "perm", "xs", "ys", "is_core", "cell_start",
             "cluster_id_per_cell", "uf", "sorted_labels_pre_border", "sorted_labels_final"]
    for k, t in zip(names, out):
        a = t.cpu().numpy()
        b = o[k]
        if k == "keys_sorted":
            b = b.view(np.int64)
        assert a.shape == b.shape, f"{name}/{k}: shape {a.shape} vs {b.shape}"
        assert np.array_equal(a, b), f"{name}/{k}: {(a != b).sum()} entries differ"


def _to_input_order(perm, sorted_vals):
    out = np.empty_like(sorted_vals)
    out[perm] = sorted_vals
    return out


@pytest.mark.parametrize("name,X,eps,ms", CASES, ids=IDS)
def test_counting_sort_intermediates(name, X, eps, ms):
    """The plain call's counting sort (dense key spaces) places the points of
    a cell in arrival order, not the reference's stable order. Every
    order-free intermediate must still equal the oracle's: the sorted keys,
    the cells, cluster id per cell, union-find roots and every label; the
    points of each cell are the same set; per-point values (sorted
    coordinates, core flags, sorted labels) equal the oracle's once mapped to
    input order through perm."""
    Xd = torch.from_numpy(X).cuda()
    _, info = _C.dbscan2d_info(Xd, eps, ms)
    if info["passes"] != 0:
        pytest.skip("sparse key space: the plain call takes the radix sort")
    _check_unstable_intermediates(name, X, Xd, eps, ms)


@pytest.mark.parametrize("n", [1_000_000, 400_000])
def test_counting_sort_intermediates_large(n):
    """The same order-free checks on clouds of 10^5 - 10^6 points."""
    X = synthetic.constant_density(n, seed=4) if n >= 10**6 else datasets.dense_overlapping_blobs(n, 3)
    Xd = torch.from_numpy(X).cuda()
    _, info = _C.dbscan2d_info(Xd, 0.5, 10)
    assert info["sort_form"] == 1, info
    _check_unstable_intermediates(f"dense_{n}", X, Xd, 0.5, 10)


def _check_unstable_intermediates(name, X, Xd, eps, ms):
    out = _C.dbscan2d_cuda_debug(Xd, eps, ms, stable_sort=False)
    names = ["labels", "keys_sorted", "perm", "xs", "ys", "is_core", "cell_start",
             "cluster_id_per_cell", "uf", "sorted_labels_pre_border", "sorted_labels_final"]
    d = {k: t.cpu().numpy() for k, t in zip(names, out)}
    o = oracle.dbscan2d(X, eps, ms, debug=True)
    for k in ("labels", "cell_start", "cluster_id_per_cell", "uf"):
        assert np.array_equal(d[k], o[k]), f"{name}/{k}: {(d[k] != o[k]).sum()} entries differ"
    assert np.array_equal(d["keys_sorted"], o["keys_sorted"].view(np.int64)), f"{name}/keys_sorted"
    n = X.shape[0]
    perm = d["perm"]
    assert np.array_equal(np.sort(perm), np.arange(n)), f"{name}: perm is not a permutation"
    cs = d["cell_start"]
    cell_of = np.repeat(np.arange(cs.size - 1), np.diff(cs))
    mine = perm[np.lexsort((perm, cell_of))]
    theirs = o["perm"][np.lexsort((o["perm"], cell_of))]
    assert np.array_equal(mine, theirs), f"{name}: cells hold different points"
    xs, ys = d["xs"], d["ys"]
    assert np.array_equal(xs.view(np.uint32), X[perm, 0].view(np.uint32)), f"{name}/xs"
    assert np.array_equal(ys.view(np.uint32), X[perm, 1].view(np.uint32)), f"{name}/ys"
    for k in ("is_core", "sorted_labels_pre_border", "sorted_labels_final"):
        a = _to_input_order(perm, d[k])
        b = _to_input_order(o["perm"], o[k])
        assert np.array_equal(a, b), f"{name}/{k}: {(a != b).sum()} points differ"


def test_repeated_runs_bit_identical():
    for make in (datasets.dense_overlapping_blobs, datasets.near_percolation_uniform):
        X = torch.from_numpy(make(50_000, 0)).cuda()
        first = dbscan2d(X, 0.5, 5)
        for _ in range(4):
            assert torch.equal(first, dbscan2d(X, 0.5, 5))


def test_batched_equals_plain():
    rng = np.random.default_rng(5)
    clouds, eps, ms = [], [], []
    for k in range(37):
        n = int(rng.integers(1, 3000)) if k % 5 else 0
        clouds.append(datasets.dense_overlapping_blobs(max(n, 0), k) if n else np.zeros((0, 2), np.float32))
        eps.append(float(rng.uniform(0.2, 1.0)))
        ms.append(int(rng.integers(1, 33)))
    off = np.concatenate([[0], np.cumsum([c.shape[0] for c in clouds])])
    X = torch.from_numpy(np.concatenate(clouds)).cuda()
    lab = dbscan2d_batched(X, off, eps, ms).cpu().numpy()
    for s, c in enumerate(clouds):
        if c.shape[0] == 0:
            continue
        want = oracle.dbscan2d(c, eps[s], ms[s])
        got = lab[off[s]:off[s + 1]]
        assert np.array_equal(got, want), f"cloud {s}: {(got != want).sum()} labels differ"


def test_cpu_tensor_roundtrip():
    X = datasets.three_blobs()
    lab = dbscan2d(torch.from_numpy(X), 1.0, 5)
    assert lab.device.type == "cpu" and lab.dtype == torch.int32
    assert np.array_equal(lab.numpy(), oracle.dbscan2d(X, 1.0, 5))


@pytest.mark.parametrize("name,X,eps,ms", CASES, ids=IDS)
def test_labels_match_reference_cuda(name, X, eps, ms):
    ref = refmod.load("cuda")
    if ref is None:
        pytest.skip("reference CUDA build not present in oracle/_ref/cuda")
    want = ref.dbscan2d(torch.from_numpy(X).cuda(), eps, ms).cpu().numpy()
    ours = dbscan2d(torch.from_numpy(X).cuda(), eps, ms).cpu().numpy()
    diff = np.flatnonzero(ours != want)
    assert diff.size == 0, f"{name}: {diff.size} labels differ from the reference CUDA path"


def test_graph_replay_across_sizes():
    """Plain calls on CUDA tensors replay one cached graph per device, updated
    call by call (new pointers, new grid sizes). Alternating sizes, and a
    sparse cloud (radix path) between dense ones, keep the oracle's labels."""
    rng = np.random.default_rng(21)
    clouds = []
    for n in (1, 5, 1000, 50_000, 3, 200_000, 700):
        clouds.append(datasets.three_blobs(n) if n >= 10 else rng.normal(0, 1, (n, 2)).astype(np.float32))
    sparse = rng.uniform(-3000, 3000, size=(20_000, 2)).astype(np.float32)
    seq = clouds + [sparse] + clouds[::-1]
    for X in seq:
        got = dbscan2d(torch.from_numpy(X).cuda(), 0.5, 4).cpu().numpy()
        assert np.array_equal(got, oracle.dbscan2d(X, 0.5, 4)), X.shape
