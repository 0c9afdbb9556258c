"""The reference's own test suite (ryanirl/dbscan-torch v0.2.0 tests/), run
against this build. Same inputs, same assertions, same tolerances:

  test_basic.py          smoke, empty, all noise, single point, min_samples > N,
                         non-contiguous input, output device, sklearn parity
  test_sklearn_parity.py six sklearn datasets: exact cluster count, ARI >= 0.99
  test_determinism.py    bit-identical labels over repeated runs
  test_eps_boundary.py   merge iff the float32 rule; brute-force parity
  test_class_wrapper.py  numpy/torch in-out contract of the DBSCAN class

The reference parametrises over "cpu" and "cuda"; here both devices run the
same CUDA pipeline ("cpu" = host tensors copied to the GPU and back), so the
whole module needs a GPU.
"""

import numpy as np
import pytest
import torch

import datasets
from conftest import canonical
from dbscan_torch import DBSCAN, dbscan2d

pytestmark = pytest.mark.gpu

DEVICES = ["cpu", "cuda"]


# ------------------------------------------------------------- test_basic
def test_three_blobs():
    X = torch.from_numpy(datasets.three_blobs())
    labels = dbscan2d(X, eps=1.0, min_samples=5)
    assert labels.dtype == torch.int32 and labels.shape == (X.shape[0],)
    assert len(set(labels.tolist()) - {-1}) == 3
    assert (labels == -1).sum().item() < 0.05 * X.shape[0]


@pytest.mark.parametrize("device", DEVICES)
def test_empty(device):
    labels = dbscan2d(torch.empty((0, 2), dtype=torch.float32, device=device), eps=1.0, min_samples=5)
    assert labels.shape == (0,) and labels.device.type == device


@pytest.mark.parametrize("device", DEVICES)
def test_all_noise(device):
    X = (torch.arange(20, dtype=torch.float32) * 100.0).unsqueeze(1).repeat(1, 2).to(device)
    assert (dbscan2d(X, eps=1.0, min_samples=2) == -1).all()


@pytest.mark.parametrize("device", DEVICES)
def test_single_point(device):
    X = torch.tensor([[1.0, 2.0]], dtype=torch.float32, device=device)
    assert dbscan2d(X, eps=1.0, min_samples=1).tolist() == [0]
    assert dbscan2d(X, eps=1.0, min_samples=2).tolist() == [-1]


@pytest.mark.parametrize("device", DEVICES)
def test_min_samples_exceeds_n(device):
    X = torch.from_numpy(datasets.three_blobs(n_per=10)).to(device)
    assert (dbscan2d(X, eps=1.0, min_samples=10_000) == -1).all()


@pytest.mark.parametrize("device", DEVICES)
def test_non_contiguous_input(device):
    X = torch.from_numpy(datasets.three_blobs()).to(device)
    Xv = X[::2]
    assert not Xv.is_contiguous()
    assert torch.equal(dbscan2d(Xv, eps=1.0, min_samples=5), dbscan2d(Xv.contiguous().clone(), 1.0, 5))


@pytest.mark.parametrize("device", DEVICES)
def test_output_device_matches_input(device):
    X = torch.from_numpy(datasets.three_blobs()).to(device)
    assert dbscan2d(X, eps=1.0, min_samples=5).device == X.device


def test_sklearn_parity_three_blobs():
    sklearn = pytest.importorskip("sklearn.cluster")
    X = torch.from_numpy(datasets.three_blobs(n_per=300, seed=42))
    ours = dbscan2d(X.cuda(), eps=0.6, min_samples=5).cpu().numpy()
    theirs = sklearn.DBSCAN(eps=0.6, min_samples=5).fit_predict(X.numpy())
    assert (canonical(ours) != canonical(theirs)).sum() <= 0.01 * X.shape[0]


def test_host_and_device_inputs_agree():
    X = torch.from_numpy(datasets.three_blobs(n_per=500, seed=7))
    a = dbscan2d(X, eps=0.6, min_samples=5)
    b = dbscan2d(X.cuda(), eps=0.6, min_samples=5).cpu()
    assert torch.equal(a, b)


# ---------------------------------------------------- test_sklearn_parity
@pytest.mark.parametrize("device", DEVICES)
@pytest.mark.parametrize("name,X,eps,ms", datasets.sklearn_like(), ids=[c[0] for c in datasets.sklearn_like()])
def test_sklearn_datasets(device, name, X, eps, ms):
    from sklearn.cluster import DBSCAN as SklearnDBSCAN
    from sklearn.metrics import adjusted_rand_score
    X = np.asarray(X, dtype=np.float32)
    ours = dbscan2d(torch.from_numpy(X).to(device), eps=eps, min_samples=ms).cpu().numpy()
    theirs = SklearnDBSCAN(eps=eps, min_samples=ms).fit_predict(X)
    n_ours = int(ours.max()) + 1 if (ours >= 0).any() else 0
    n_theirs = int(theirs.max()) + 1 if (theirs >= 0).any() else 0
    assert n_ours == n_theirs
    assert adjusted_rand_score(theirs, ours) >= 0.99


@pytest.mark.parametrize("device", DEVICES)
def test_single_giant_cluster(device):
    X = np.random.default_rng(0).normal(0.0, 0.3, size=(2000, 2)).astype(np.float32)
    labels = dbscan2d(torch.from_numpy(X).to(device), eps=0.5, min_samples=5).cpu().numpy()
    assert int(labels.max()) + 1 == 1 and (labels == -1).sum() == 0


# ------------------------------------------------------- test_determinism
@pytest.mark.parametrize("device", DEVICES)
@pytest.mark.parametrize("make", [datasets.dense_overlapping_blobs, datasets.near_percolation_uniform],
                         ids=["dense_blobs", "uniform"])
def test_repeated_runs_bit_identical(device, make):
    X = torch.from_numpy(make(50_000, 0)).to(device)
    first = dbscan2d(X, eps=0.5, min_samples=5)
    for _ in range(2):
        assert torch.equal(first, dbscan2d(X, eps=0.5, min_samples=5))


# ------------------------------------------------------ test_eps_boundary
def _boundary_float(eps, cell, side):
    inv_r = np.float32(np.sqrt(np.float32(2.0))) / np.float32(eps)
    x = np.float32(cell + (1 if side == "high" else 0)) / inv_r
    step = np.float32(-np.inf) if side == "high" else np.float32(np.inf)
    while int(np.floor(x * inv_r)) != cell:
        x = np.nextafter(x, step)
    while int(np.floor(np.nextafter(x, -step) * inv_r)) == cell:
        x = np.nextafter(x, -step)
    return float(x)


_C0H, _C2L = _boundary_float(1.0, 0, "high"), _boundary_float(1.0, 2, "low")
_OVER = float(np.nextafter(np.float32(1.5), np.float32(2.0)))
_UNDER = float(np.nextafter(np.float32(1.5), np.float32(0.0)))


@pytest.mark.parametrize("device", DEVICES)
@pytest.mark.parametrize("a,b", [((0.5, 0.5), (1.5, 0.5)), ((0.5, 0.5), (_OVER, 0.5)),
                                 ((0.5, 0.5), (_UNDER, 0.5)), ((_C0H, _C0H), (_C2L, _C2L))],
                         ids=["exact_eps_ring2_axis", "one_ulp_over", "one_ulp_under", "ring2_diagonal_corner"])
def test_merge_follows_float32_rule(device, a, b):
    X = torch.from_numpy(np.array([a] * 5 + [b] * 5, dtype=np.float32)).to(device)
    labels = dbscan2d(X, eps=1.0, min_samples=5).cpu()
    ex = np.float32(b[0]) - np.float32(a[0])
    ey = np.float32(b[1]) - np.float32(a[1])
    expected = 1 if bool(ex * ex + ey * ey <= np.float32(1.0)) else 2
    assert (labels >= 0).all()
    assert len(set(labels.tolist()) - {-1}) == expected


@pytest.mark.parametrize("device", DEVICES)
def test_bruteforce_parity_dense(device):
    from test_oracle import _bruteforce
    rng = np.random.default_rng(7)
    centers = rng.uniform(-4.0, 4.0, size=(8, 2)).astype(np.float32)
    X = np.concatenate([rng.normal(c, 1.0, size=(150, 2)).astype(np.float32) for c in centers])
    rng.shuffle(X)
    ours = dbscan2d(torch.from_numpy(X).to(device), eps=0.35, min_samples=5).cpu().numpy()
    assert int((canonical(ours) != canonical(_bruteforce(X, 0.35, 5))).sum()) == 0


# ----------------------------------------------------- test_class_wrapper
def test_numpy_in_numpy_out():
    X = datasets.three_blobs()
    clf = DBSCAN(eps=1.0, min_samples=5).fit(X)
    assert isinstance(clf.labels_, np.ndarray) and clf.labels_.shape == (X.shape[0],)
    assert len(set(clf.labels_.tolist()) - {-1}) == 3


@pytest.mark.parametrize("device", DEVICES)
def test_torch_in_torch_out(device):
    X = torch.from_numpy(datasets.three_blobs()).to(device)
    clf = DBSCAN(eps=1.0, min_samples=5).fit(X)
    assert isinstance(clf.labels_, torch.Tensor) and clf.labels_.dtype == torch.int32
    assert clf.labels_.device == X.device


def test_fit_returns_self_and_fit_predict():
    X = datasets.three_blobs()
    clf = DBSCAN(eps=1.0, min_samples=5)
    assert clf.fit(X) is clf
    np.testing.assert_array_equal(DBSCAN(eps=1.0, min_samples=5).fit_predict(X), clf.labels_)


def test_float64_input_is_cast_and_y_ignored():
    X = torch.from_numpy(datasets.three_blobs()).to(torch.float64)
    clf = DBSCAN(eps=1.0, min_samples=5).fit(X)
    assert clf.labels_.shape == (X.shape[0],)
    Xn = datasets.three_blobs()
    np.testing.assert_array_equal(DBSCAN(1.0, 5).fit_predict(Xn, np.zeros(len(Xn))),
                                  DBSCAN(1.0, 5).fit_predict(Xn))
