"""Seeded synthetic point clouds for the benchmark workloads.

The reference publishes numbers only on "synthetic 2D Gaussian clusters at
constant density" (ryanirl/dbscan-torch README.md:82-83) without the
generator; these seeded generators stand in for it with the shapes, sizes and
distributions of the five benchmark workloads:

  blobs_with_noise   N=100,000: 20 Gaussian blobs (sigma 1) with centres
                     uniform in [-50, 50]^2, equal mass, plus 5% uniform noise
                     over [-60, 60]^2 (eps 0.5, min_samples 10)
  constant_density   N in {1M, 5M, 10M}: K = N/5,000 blobs (sigma 1) with
                     centres uniform in a square of side 2*sqrt(N)/10 centred
                     at 0, plus 2% uniform noise over the same square
  adversarial        4M points: 50% uniform in a 0.2 x 0.2 square, 30% on 64
                     Archimedean spirals (arm spacing 0.3, jitter sigma 0.05),
                     20% on an integer lattice scaled by 0.5
  batch              many clouds of log-uniform size, each blobs_with_noise
                     with its own seed, eps and min_samples
  request_stream     Poisson arrivals of clouds of log-uniform size

All outputs are float32 (N, 2) numpy arrays, shuffled.
"""

from __future__ import annotations

import numpy as np
import torch


def blobs_with_noise(n: int = 100_000, seed: int = 0, n_blobs: int = 20,
                     noise_frac: float = 0.05) -> np.ndarray:
    rng = np.random.default_rng(seed)
    n_noise = int(round(n * noise_frac))
    n_blob = n - n_noise
    centers = rng.uniform(-50.0, 50.0, size=(n_blobs, 2))
    per = np.full(n_blobs, n_blob // n_blobs)
    per[: n_blob - per.sum()] += 1
    parts = [rng.normal(centers[i], 1.0, size=(per[i], 2)) for i in range(n_blobs)]
    parts.append(rng.uniform(-60.0, 60.0, size=(n_noise, 2)))
    X = np.concatenate(parts).astype(np.float32)
    rng.shuffle(X)
    return X


def constant_density(n: int = 10_000_000, seed: int = 0, noise_frac: float = 0.02) -> np.ndarray:
    rng = np.random.default_rng(seed)
    k = max(1, n // 5_000)
    side = 2.0 * np.sqrt(n) / 10.0
    n_noise = int(round(n * noise_frac))
    n_blob = n - n_noise
    centers = rng.uniform(-side / 2, side / 2, size=(k, 2))
    which = np.repeat(np.arange(k), n_blob // k)
    extra = n_blob - which.size
    if extra:
        which = np.concatenate([which, np.arange(extra) % k])
    X = np.empty((n, 2), dtype=np.float32)
    X[:n_blob] = (centers[which] + rng.standard_normal((n_blob, 2))).astype(np.float32)
    X[n_blob:] = rng.uniform(-side / 2, side / 2, size=(n_noise, 2)).astype(np.float32)
    rng.shuffle(X)
    return X


def sparse_uniform(n: int, seed: int = 0) -> np.ndarray:
    """n points uniform over a square of side 3*sqrt(n): about 0.014 points per
    cell at eps 0.5, a key range ~70 times the point count, so the pipeline
    takes its radix sort (the profile workload of that path)."""
    rng = np.random.default_rng(seed)
    side = 3.0 * np.sqrt(n)
    return rng.uniform(-side / 2, side / 2, size=(n, 2)).astype(np.float32)


def adversarial(n: int = 4_000_000, seed: int = 0) -> np.ndarray:
    """Dense square at (-20, -20); 64 spirals on an 8 x 8 grid of centres
    10 apart starting at (0, 0); lattice at x >= 100. Components are >= 5
    apart, so no stencil window reaches from one to another."""
    rng = np.random.default_rng(seed)
    n_sq = n // 2
    n_sp = (n * 3) // 10
    n_lat = n - n_sq - n_sp
    sq = rng.uniform(0.0, 0.2, size=(n_sq, 2)) + np.array([-20.0, -20.0])
    # 64 Archimedean spirals r = r0 + 0.3 * theta / (2 pi), 10 turns each.
    per = np.full(64, n_sp // 64)
    per[: n_sp - per.sum()] += 1
    sp = []
    for s in range(64):
        cx, cy = (s % 8) * 10.0, (s // 8) * 10.0
        th = rng.uniform(0.0, 10 * 2 * np.pi, size=per[s])
        r = 0.5 + 0.3 * th / (2 * np.pi)
        pts = np.stack([cx + r * np.cos(th), cy + r * np.sin(th)], axis=1)
        sp.append(pts + rng.normal(0.0, 0.05, size=pts.shape))
    sp = np.concatenate(sp)
    side = int(np.ceil(np.sqrt(n_lat)))
    idx = np.arange(n_lat)
    lat = np.stack([100.0 + 0.5 * (idx % side), 0.5 * (idx // side)], axis=1)
    X = np.concatenate([sq, sp, lat]).astype(np.float32)
    rng.shuffle(X)
    return X


def batch(n_clouds: int = 4096, seed: int = 0, n_min: int = 256, n_max: int = 262_144,
          eps_range=(0.2, 1.0), ms_range=(4, 32)):
    """Returns (clouds, eps, min_samples): list of float32 (N_i, 2) arrays,
    float64 eps_i uniform in eps_range, int64 min_samples_i uniform in
    ms_range (inclusive)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(n_min), np.log(n_max), size=n_clouds)).astype(np.int64)
    eps = rng.uniform(eps_range[0], eps_range[1], size=n_clouds)
    ms = rng.integers(ms_range[0], ms_range[1] + 1, size=n_clouds)
    seeds = rng.integers(0, 2**31 - 1, size=n_clouds)
    clouds = [blobs_with_noise(int(sizes[i]), int(seeds[i])) for i in range(n_clouds)]
    return clouds, eps, ms


def batch_layout(n_clouds: int = 4096, seed: int = 0, n_min: int = 256, n_max: int = 262_144,
                 eps_range=(0.2, 1.0), ms_range=(4, 32)):
    """Sizes, eps and min_samples of the batched workload without the points
    (for the device generator): sizes log-uniform in [n_min, n_max] (int64),
    eps_i uniform in eps_range, min_samples_i uniform integers in ms_range
    (inclusive). Same draws, in the same order, as ``batch``."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(n_min), np.log(n_max), size=n_clouds)).astype(np.int64)
    eps = rng.uniform(eps_range[0], eps_range[1], size=n_clouds)
    ms = rng.integers(ms_range[0], ms_range[1] + 1, size=n_clouds)
    return sizes, eps, ms


def request_stream(rate_hz: float = 2000.0, duration_s: float = 60.0, seed: int = 0,
                   n_min: int = 1_000, n_max: int = 2_000_000, eps_range=(0.1, 1.0),
                   ms_range=(4, 32)):
    """Poisson arrivals: returns (arrival_s, sizes, eps, min_samples, seeds)."""
    rng = np.random.default_rng(seed)
    n_req = rng.poisson(rate_hz * duration_s)
    arrivals = np.sort(rng.uniform(0.0, duration_s, size=n_req))
    sizes = np.exp(rng.uniform(np.log(n_min), np.log(n_max), size=n_req)).astype(np.int64)
    eps = rng.uniform(eps_range[0], eps_range[1], size=n_req)
    ms = rng.integers(ms_range[0], ms_range[1] + 1, size=n_req)
    seeds = rng.integers(0, 2**31 - 1, size=n_req)
    return arrivals, sizes, eps, ms, seeds


def blobs_with_noise_device(sizes, seed: int = 0, device="cuda", n_blobs: int = 20,
                            noise_frac: float = 0.05):
    """Many clouds with the distribution of ``blobs_with_noise``, generated on
    the device in one pass (the numpy generator's row shuffle takes minutes
    for ~10^8 points). Cloud k has ``sizes[k]`` points: ``n_blobs`` Gaussian
    blobs (sigma 1) with centres uniform in [-50, 50]^2 and equal mass (the
    first ``n_blob % n_blobs`` blobs one point larger), plus
    ``round(noise_frac * n)`` uniform points over [-60, 60]^2, shuffled within
    the cloud. Seeded (torch's device generator), so repeatable on one GPU
    type; the random streams differ from the numpy generator's.

    Returns (X float32 (sum(sizes), 2) on ``device``, offsets int64 (S + 1,)
    on the host)."""
    dev = torch.device(device)
    sizes = torch.as_tensor(np.asarray(sizes, dtype=np.int64))
    S = sizes.numel()
    off = torch.zeros(S + 1, dtype=torch.int64)
    off[1:] = torch.cumsum(sizes, 0)
    N = int(off[-1])
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))
    sizes_d = sizes.to(dev)
    cloud = torch.repeat_interleave(torch.arange(S, device=dev), sizes_d)
    j = torch.arange(N, device=dev) - off.to(dev)[cloud]
    n_noise = torch.round(sizes_d.double() * noise_frac).long()
    n_blob = sizes_d - n_noise
    per = n_blob // n_blobs
    rem = n_blob - per * n_blobs
    boundary = rem * (per + 1)
    jb = j
    blob = torch.where(jb < boundary[cloud], jb // (per[cloud] + 1),
                       rem[cloud] + (jb - boundary[cloud]) // per[cloud].clamp(min=1))
    blob = blob.clamp(max=n_blobs - 1)
    centers = torch.rand((S, n_blobs, 2), generator=g, device=dev, dtype=torch.float64) * 100.0 - 50.0
    pts = centers[cloud, blob] + torch.randn((N, 2), generator=g, device=dev, dtype=torch.float64)
    noise = torch.rand((N, 2), generator=g, device=dev, dtype=torch.float64) * 120.0 - 60.0
    X = torch.where((j < n_blob[cloud])[:, None], pts, noise).to(torch.float32)
    del pts, noise, blob, jb
    key = cloud.double() + torch.rand(N, generator=g, device=dev, dtype=torch.float64)
    order = torch.argsort(key)
    return X[order].contiguous(), off
