"""CPU checks of the oracle (oracle/dbscan_oracle.c) before it is trusted.

Pinned against:
  * the reference's own known-answer tests, read from its test files:
    test_basic.py:54-91 (empty, all noise, single point, min_samples > N),
    test_eps_boundary.py:191-247 (exact eps, +-1 ulp, ring-2 diagonal corner:
    merge iff the float32 rule says so) and :254-326 (brute-force DBSCAN with
    the CUDA tie rule, exact after canonical relabelling);
  * the reference's CPU implementation built from its sources
    (oracle/_ref/cpu): same core set and same partition up to border ties and
    the order of cluster ids (the CPU path numbers cells in signed order and
    breaks border ties by scan order, dbscan_grid.hpp:176-178, :425-437);
  * golden labels produced by the reference's CUDA build on a B200
    (tests/golden/, see make_golden.py): bit-exact.
"""

import glob
import os

import numpy as np
import pytest
import torch

import datasets
import oracle
import refmod
from conftest import canonical

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


# ----------------------------------------------------------- KATs (test_basic)
def test_empty():
    assert oracle.dbscan2d(np.zeros((0, 2), np.float32), 1.0, 5).shape == (0,)


def test_all_noise():
    X = (np.arange(20, dtype=np.float32) * 100.0)[:, None].repeat(2, 1)
    assert (oracle.dbscan2d(X, 1.0, 2) == -1).all()


def test_single_point():
    X = np.array([[1.0, 2.0]], np.float32)
    assert oracle.dbscan2d(X, 1.0, 1).tolist() == [0]
    assert oracle.dbscan2d(X, 1.0, 2).tolist() == [-1]


def test_min_samples_exceeds_n():
    assert (oracle.dbscan2d(datasets.three_blobs(10), 1.0, 10_000) == -1).all()


def test_three_blobs():
    lab = oracle.dbscan2d(datasets.three_blobs(), 1.0, 5)
    assert len(set(lab.tolist()) - {-1}) == 3
    assert (lab == -1).sum() < 0.05 * lab.size


# ---------------------------------------------------- eps boundary (KATs)
_EPS, _MS = 1.0, 5


def _boundary_float(eps, cell, side):
    inv_r = np.float32(np.sqrt(np.float32(2.0))) / np.float32(eps)
    x = np.float32(cell + (1 if side == "high" else 0)) / inv_r
    step = np.float32(-np.inf) if side == "high" else np.float32(np.inf)
    while int(np.floor(x * inv_r)) != cell:
        x = np.nextafter(x, step)
    while int(np.floor(np.nextafter(x, -step) * inv_r)) == cell:
        x = np.nextafter(x, -step)
    return float(x)


_C0H = _boundary_float(_EPS, 0, "high")
_C2L = _boundary_float(_EPS, 2, "low")
_OVER = float(np.nextafter(np.float32(1.5), np.float32(2.0)))
_UNDER = float(np.nextafter(np.float32(1.5), np.float32(0.0)))
BOUNDARY = [((0.5, 0.5), (1.5, 0.5)), ((0.5, 0.5), (_OVER, 0.5)), ((0.5, 0.5), (_UNDER, 0.5)),
            ((_C0H, _C0H), (_C2L, _C2L))]


def _rule(a, b, eps):
    ex = np.float32(b[0]) - np.float32(a[0])
    ey = np.float32(b[1]) - np.float32(a[1])
    return bool(ex * ex + ey * ey <= np.float32(eps) * np.float32(eps))


@pytest.mark.parametrize("a,b", BOUNDARY, ids=["exact", "ulp_over", "ulp_under", "corner"])
def test_merge_follows_float32_rule(a, b):
    X = np.array([a] * _MS + [b] * _MS, np.float32)
    lab = oracle.dbscan2d(X, _EPS, _MS)
    assert (lab >= 0).all()
    assert len(set(lab.tolist())) == (1 if _rule(a, b, _EPS) else 2)


def _bruteforce(X, eps, ms):
    """Restatement of test_eps_boundary.py:254-294 (inclusive float32 eps,
    counts include self, borders to the nearest core, ties to smaller index)."""
    ex = X[:, 0][None, :] - X[:, 0][:, None]
    ey = X[:, 1][None, :] - X[:, 1][:, None]
    d2 = ex * ex + ey * ey
    within = d2 <= np.float32(eps) * np.float32(eps)
    core = within.sum(1) >= ms
    parent = list(range(len(X)))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    ci = np.flatnonzero(core)
    for i in ci:
        for j in np.flatnonzero(within[i] & core):
            a, b = find(int(i)), find(int(j))
            if a != b:
                parent[max(a, b)] = min(a, b)
    lab = np.full(len(X), -1, np.int32)
    ids = {}
    for i in ci:
        lab[i] = ids.setdefault(find(int(i)), len(ids))
    for i in np.flatnonzero(~core):
        cand = np.flatnonzero(within[i] & core)
        if cand.size:
            lab[i] = lab[cand[np.lexsort((cand, d2[i, cand]))[0]]]
    return lab


def test_bruteforce_parity_dense():
    rng = np.random.default_rng(7)
    centers = rng.uniform(-4.0, 4.0, size=(8, 2)).astype(np.float32)
    X = np.concatenate([rng.normal(c, 1.0, size=(150, 2)).astype(np.float32) for c in centers])
    rng.shuffle(X)
    ours = oracle.dbscan2d(X, 0.35, 5, forms=(oracle.FORM_UNFUSED,) * 7)
    assert np.array_equal(canonical(ours), canonical(_bruteforce(X, 0.35, 5)))


# ------------------------------------------- reference CPU path (built here)
REF_CASES = [c for c in datasets.parity_cases() if c[0] not in ("huge_coords", "wide_sparse")]


@pytest.mark.parametrize("name,X,eps,ms", REF_CASES, ids=[c[0] for c in REF_CASES])
def test_against_reference_cpu(name, X, eps, ms):
    ref = refmod.load("cpu")
    if ref is None:
        pytest.skip("reference CPU build not present in oracle/_ref/cpu")
    want = ref.dbscan2d(torch.from_numpy(X), eps, ms).numpy()
    got = oracle.dbscan2d(X, eps, ms, forms=(oracle.FORM_UNFUSED,) * 7)
    # Same noise set; same partition of the points that are core in both.
    assert np.array_equal(got == -1, want == -1), name
    dbg = oracle.dbscan2d(X, eps, ms, debug=True, forms=(oracle.FORM_UNFUSED,) * 7)
    core = np.zeros(X.shape[0], bool)
    core[dbg["perm"]] = dbg["is_core"].astype(bool)
    assert np.array_equal(canonical(got[core]), canonical(want[core])), name


# ------------------------------------------------------------ golden labels
GOLDEN_FILES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


@pytest.mark.parametrize("path", GOLDEN_FILES, ids=[os.path.basename(p) for p in GOLDEN_FILES])
def test_golden_reference_cuda(path):
    g = np.load(path)
    X, eps, ms = g["X"], float(g["eps"]), int(g["min_samples"])
    got = oracle.dbscan2d(X, eps, ms, debug="perm" in g.files)
    if isinstance(got, dict):
        for k in ("perm", "is_core", "cell_start", "cluster_id_per_cell", "uf",
                  "sorted_labels_pre_border", "sorted_labels_final"):
            if k in g.files:
                assert np.array_equal(got[k], g[k]), f"{k} differs"
        got = got["labels"]
    assert np.array_equal(got, g["labels"])
