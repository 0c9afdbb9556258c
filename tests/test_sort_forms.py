"""The sort step on key spaces of every size class, against the oracle
(bit-exact labels).

Points sit in W = wx * 2^ceil(log2 wy) compacted cell keys (cell side
eps / sqrt(2)). A dense key space (W <= 6N + 4096) takes the counting sort
over keys, whose per-key counters, scan and dense cell map all scale with W;
a sparse one takes the radix sort. The clouds below cover W from under a
million keys to 18 million, a sparse key space, a cloud with most points in
a few cells, and many dense clouds in one batched run; `passes` from the
plan read-back tells dense (0) from radix.
"""

import numpy as np
import pytest
import torch

import oracle
from dbscan_torch import _C, BatchedPlan, dbscan2d, dbscan2d_batched, synthetic

pytestmark = pytest.mark.gpu

EPS = 0.5
SIDE = EPS / np.sqrt(2.0)  # cell side


def _rect(n, wx, wy, seed):
    """n uniform points over about wx x wy cells."""
    rng = np.random.default_rng(seed)
    X = np.empty((n, 2), np.float32)
    X[:, 0] = rng.uniform(0.0, wx * SIDE, n)
    X[:, 1] = rng.uniform(0.0, wy * SIDE, n)
    return X


FORMS = [
    # name, X, min_samples, dense
    ("dense_W0.9M", _rect(300_000, 849, 849, 1), 3, True),
    ("dense_W1.5M", _rect(500_000, 1500, 1000, 2), 3, True),
    ("dense_W4.1M", _rect(1_200_000, 2000, 2000, 3), 3, True),
    ("dense_W18M", _rect(5_000_000, 4500, 4000, 4), 3, True),
    ("radix_sparse", _rect(100_000, 3000, 3000, 5), 2, False),     # W ~ 12M > 6N + 4096
    ("hot_cell", synthetic.adversarial(400_000, seed=6), 4, True),  # half the points in a few cells
]


@pytest.mark.parametrize("name,X,ms,dense", FORMS, ids=[f[0] for f in FORMS])
def test_sort_form_matches_oracle(name, X, ms, dense):
    Xd = torch.from_numpy(X).cuda()
    ours, info = _C.dbscan2d_info(Xd, EPS, ms)
    assert (info["passes"] == 0) == dense, info
    want = oracle.dbscan2d(X, EPS, ms)
    got = ours.cpu().numpy()
    diff = np.flatnonzero(got != want)
    assert diff.size == 0, f"{name}: {diff.size}/{X.shape[0]} labels differ"
    # A second run on the same workspace layout gives the same labels.
    assert np.array_equal(dbscan2d(Xd, EPS, ms).cpu().numpy(), want)


def test_batched_pooled_budget():
    """A batch whose clouds are sparse on their own (key range above 6N + 4096
    each) but fit the summed budget takes the counting sort over one pooled
    map; labels per cloud equal plain calls (which take the radix sort)."""
    rng = np.random.default_rng(9)
    dense = [synthetic.constant_density(200_000, seed=k) for k in range(3)]
    sparse = [rng.uniform(-40, 40, size=(300, 2)).astype(np.float32) for _ in range(5)]
    clouds = dense[:1] + sparse[:2] + dense[1:] + sparse[2:]
    X = np.concatenate(clouds)
    off = np.concatenate([[0], np.cumsum([len(c) for c in clouds])])
    Xd = torch.from_numpy(X).cuda()
    lab = dbscan2d_batched(Xd, off.tolist(), 0.5, 4).cpu().numpy()
    # The same batch through a plan: one pooled map, the counting sort.
    plan = BatchedPlan(off.tolist())
    assert np.array_equal(plan.run(Xd, 0.5, 4).cpu().numpy(), lab)
    st = plan.stats()
    assert st["sort_form"] == 1, st
    for k, c in enumerate(clouds):
        want = oracle.dbscan2d(c, 0.5, 4)
        assert np.array_equal(lab[off[k]:off[k + 1]], want), f"cloud {k}"
        plain = dbscan2d(torch.from_numpy(c).cuda(), 0.5, 4).cpu().numpy()
        assert np.array_equal(plain, want)


def test_batched_dense_clouds():
    """Many dense clouds in one run: a thread's run of points crosses clouds,
    so the per-cloud key parameters change inside the sort's point loops."""
    rng = np.random.default_rng(7)
    sizes = rng.integers(1, 20_000, size=60)
    sizes[[3, 17]] = 0  # empty clouds in between
    clouds = [synthetic.blobs_with_noise(int(s), seed=100 + k, n_blobs=3) if s else
              np.zeros((0, 2), np.float32) for k, s in enumerate(sizes)]
    eps = rng.uniform(0.3, 1.5, size=len(clouds))
    ms = rng.integers(2, 12, size=len(clouds))
    X = np.concatenate(clouds).astype(np.float32)
    off = np.concatenate([[0], np.cumsum(sizes)])
    lab = dbscan2d_batched(torch.from_numpy(X).cuda(), off.tolist(), eps.tolist(), ms.tolist()).cpu().numpy()
    for k in range(len(clouds)):
        want = oracle.dbscan2d(clouds[k], float(eps[k]), int(ms[k]))
        assert np.array_equal(lab[off[k]:off[k + 1]], want), f"cloud {k}"


def _with_specials(kind, seed):
    X = synthetic.blobs_with_noise(60_000, seed=seed, n_blobs=6)
    rng = np.random.default_rng(seed)
    idx = rng.choice(X.shape[0], size=40, replace=False)
    if kind == "nan":
        X[idx[:20], 0] = np.nan
        X[idx[20:], 1] = np.nan
    else:
        X[idx[:20], 0] = np.inf
        X[idx[20:], 1] = -np.inf
    return X


@pytest.mark.parametrize("kind", ["nan", "inf"])
def test_special_coordinates(kind):
    """Points with a NaN or infinite coordinate: cells holding them get an
    infinite box (NaN) or a huge key range (inf, radix sort); the labels stay
    those of the oracle and, when present, of the reference CUDA build."""
    import refmod
    X = _with_specials(kind, 11)
    ours = dbscan2d(torch.from_numpy(X).cuda(), EPS, 5).cpu().numpy()
    assert np.array_equal(ours, oracle.dbscan2d(X, EPS, 5))
    ref = refmod.load("cuda")
    if ref is not None:
        assert np.array_equal(ours, ref.dbscan2d(torch.from_numpy(X).cuda(), EPS, 5).cpu().numpy())


def test_batched_above_core_first_threshold():
    """More than 16M points in one run: the label pass orders its work core
    labels first (the label array is larger than L2); labels still equal a
    plain call per cloud."""
    sizes = [4_500_000, 4_500_000, 4_500_000, 4_500_000]
    X, off = synthetic.blobs_with_noise_device(sizes, seed=5, device="cuda")
    offl = off.tolist()
    eps, ms = [0.3, 0.5, 0.8, 1.0], [4, 10, 16, 32]
    lab = dbscan2d_batched(X, offl, eps, ms)
    for k in range(len(sizes)):
        want = dbscan2d(X[offl[k]:offl[k + 1]], eps[k], ms[k])
        assert torch.equal(lab[offl[k]:offl[k + 1]], want), f"cloud {k}"


@pytest.mark.parametrize("order", ["cell_order", "dominant_cell"])
def test_hot_keys(order):
    """Rows of 32 consecutive points that share a cell (hot keys) are ranked by
    the count pass through a 64-slot table. Points in cell order make nearly
    every row hot, so the table fills and later keys stay cold; a cloud with
    most points in one cell keeps one key hot. Labels equal the oracle's."""
    if order == "cell_order":
        X = synthetic.constant_density(250_000, seed=8)
        inv_r = np.float32(np.sqrt(np.float32(2.0)) / np.float32(EPS))
        kx = np.floor(X[:, 0] * inv_r).astype(np.int64)
        ky = np.floor(X[:, 1] * inv_r).astype(np.int64)
        X = X[np.lexsort((ky, kx))]
        ms = 10
    else:
        rng = np.random.default_rng(9)
        X = synthetic.blobs_with_noise(200_000, seed=9, n_blobs=5)
        X[:120_000] = rng.uniform(0.01, 0.05, size=(120_000, 2)).astype(np.float32)
        X = X[rng.permutation(X.shape[0])]
        ms = 4
    ours, info = _C.dbscan2d_info(torch.from_numpy(X).cuda(), EPS, ms)
    assert info["sort_form"] == 1, info  # the counting sort ran
    if order == "cell_order":
        # Nearly every row is hot: all 64 slots are taken and later hot keys
        # find their probe window full and stay cold.
        assert info["hot_slots"] == 64, info
    else:
        # The dominant cell's key (and few others) went through the table.
        assert 1 <= info["hot_slots"] < 64, info
    want = oracle.dbscan2d(X, EPS, ms)
    assert np.array_equal(ours.cpu().numpy(), want)


def test_spread_keys_stay_cold():
    """A shuffled constant-density cloud has no row with 8 points of one cell:
    the hot-key table stays empty, every point takes the cold path."""
    X = synthetic.constant_density(250_000, seed=8)
    ours, info = _C.dbscan2d_info(torch.from_numpy(X).cuda(), EPS, 10)
    assert info["sort_form"] == 1 and info["hot_slots"] == 0, info
    assert np.array_equal(ours.cpu().numpy(), oracle.dbscan2d(X, EPS, 10))
