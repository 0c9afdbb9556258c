"""Seeded test inputs shared by the parity tests.

Each case is (name, X float32 (N, 2), eps, min_samples), sized so the CPU
oracle finishes in well under a second. The shapes cover the reference's own
test inputs (test_basic.py:14-20, test_determinism.py:26-51,
test_sklearn_parity.py:96-119, test_eps_boundary.py:182-228) and the cases
the reference's cell layout makes delicate: clouds straddling zero in both
axes (unsigned key order), single-point cells, dense cells far above
min_samples, lattice pairs at exactly eps, huge coordinates, min_samples 1.
"""

from __future__ import annotations

import numpy as np


def three_blobs(n_per=200, seed=0, scale=0.3):
    rng = np.random.default_rng(seed)
    centers = np.array([[0.0, 0.0], [10.0, 0.0], [0.0, 10.0]], dtype=np.float32)
    return np.concatenate([rng.normal(c, scale, size=(n_per, 2)) for c in centers]).astype(np.float32)


def dense_overlapping_blobs(n, seed):
    rng = np.random.default_rng(seed)
    k = 20
    centers = rng.uniform(-25.0, 25.0, size=(k, 2)).astype(np.float32)
    per = np.full(k, n // k)
    per[: n - per.sum()] += 1
    X = np.concatenate([rng.normal(centers[c], 2.0, size=(per[c], 2)).astype(np.float32)
                        for c in range(k)])
    rng.shuffle(X)
    return X


def near_percolation_uniform(n, seed):
    rng = np.random.default_rng(seed)
    extent = 200.0 * np.sqrt(n / 1_000_000)
    return rng.uniform(-extent, extent, size=(n, 2)).astype(np.float32)


def lattice(side=40, spacing=0.5, origin=(-7.0, -3.0)):
    g = np.arange(side, dtype=np.float32) * np.float32(spacing)
    xx, yy = np.meshgrid(g, g)
    return (np.stack([xx.ravel(), yy.ravel()], axis=1) + np.float32(origin)).astype(np.float32)


def spirals(n=6000, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for s in range(4):
        th = rng.uniform(0, 6 * np.pi, size=n // 4)
        r = 0.5 + 0.3 * th / (2 * np.pi)
        c = np.array([(s % 2) * 8.0 - 4.0, (s // 2) * 8.0 - 4.0])
        pts = np.stack([c[0] + r * np.cos(th), c[1] + r * np.sin(th)], axis=1)
        out.append(pts + rng.normal(0, 0.05, size=pts.shape))
    X = np.concatenate(out).astype(np.float32)
    rng.shuffle(X)
    return X


def dense_square(n=20000, seed=0):
    rng = np.random.default_rng(seed)
    sq = rng.uniform(0.0, 0.2, size=(n, 2))
    ring = rng.uniform(-3.0, 3.0, size=(n // 10, 2))
    X = np.concatenate([sq, ring]).astype(np.float32)
    rng.shuffle(X)
    return X


def sklearn_like(seed=0):
    from sklearn.datasets import make_blobs, make_circles, make_moons
    return [
        ("blobs_500_dense", make_blobs(n_samples=500, centers=5, cluster_std=0.5, random_state=0)[0], 0.5, 5),
        ("blobs_2k_sparse", make_blobs(n_samples=2000, centers=10, cluster_std=1.5, random_state=1)[0], 0.8, 10),
        ("blobs_10k", make_blobs(n_samples=10000, centers=20, cluster_std=0.8, random_state=2)[0], 0.5, 8),
        ("moons_1k", make_moons(n_samples=1000, noise=0.05, random_state=0)[0], 0.15, 5),
        ("moons_5k", make_moons(n_samples=5000, noise=0.07, random_state=1)[0], 0.10, 5),
        ("circles_2k", make_circles(n_samples=2000, noise=0.05, random_state=0, factor=0.5)[0], 0.10, 5),
    ]


def parity_cases():
    """(name, X, eps, min_samples) for raw-label parity with the oracle."""
    rng = np.random.default_rng(1234)
    cases = [
        ("three_blobs", three_blobs(), 1.0, 5),
        ("three_blobs_eps06", three_blobs(300, 42), 0.6, 5),
        ("dense_blobs_50k", dense_overlapping_blobs(50_000, 0), 0.5, 5),
        ("uniform_50k", near_percolation_uniform(50_000, 0), 0.5, 5),
        ("uniform_ms1", near_percolation_uniform(5_000, 3), 0.5, 1),
        ("uniform_ms2", near_percolation_uniform(20_000, 4), 0.7, 2),
        ("lattice_exact_eps_ms4", lattice(), 0.5, 4),
        ("lattice_exact_eps_ms5", lattice(), 0.5, 5),
        ("lattice_exact_eps_ms6", lattice(), 0.5, 6),
        ("spirals", spirals(), 0.5, 4),
        ("dense_square_ms32", dense_square(), 0.5, 32),
        ("dense_square_ms4", dense_square(5000, 1), 0.5, 4),
        ("offset_positive", (rng.normal(0, 1.5, size=(8000, 2)) + 1000.0).astype(np.float32), 0.3, 6),
        ("offset_negative", (rng.normal(0, 1.5, size=(8000, 2)) - 1000.0).astype(np.float32), 0.3, 6),
        ("huge_coords", (rng.normal(0, 1.0, size=(4000, 2)) * 1e6).astype(np.float32), 5e4, 3),
        ("tiny_eps", (rng.normal(0, 1e-3, size=(4000, 2))).astype(np.float32), 1e-4, 4),
        ("single_point_ms1", np.array([[1.0, 2.0]], np.float32), 1.0, 1),
        ("single_point_ms2", np.array([[1.0, 2.0]], np.float32), 1.0, 2),
        ("all_noise", ((np.arange(50, dtype=np.float32) * 100.0)[:, None].repeat(2, 1)), 1.0, 2),
        ("two_points_same_cell", np.array([[0.1, 0.1], [0.2, 0.2]], np.float32), 1.0, 2),
        ("ms_exceeds_n", three_blobs(10, 0), 1.0, 10_000),
        ("duplicates", np.repeat(rng.uniform(-2, 2, size=(300, 2)).astype(np.float32), 7, axis=0), 0.2, 5),
        ("line_x", np.stack([np.linspace(-50, 50, 20000), np.zeros(20000)], 1).astype(np.float32), 0.01, 3),
        ("wide_sparse", rng.uniform(-1e5, 1e5, size=(3000, 2)).astype(np.float32), 2.0, 2),
    ]
    for name, X, eps, ms in sklearn_like():
        cases.append((name, np.asarray(X, dtype=np.float32), eps, ms))
    return cases
