"""The plain path against the reference's CUDA path on the same B200.

Times dbscan2d on the 10M-point constant-density cloud (eps 0.5,
min_samples 10) for this build and for the reference's own CUDA build
(oracle/_ref/cuda), both through their Python entry points with the input
resident on the device, CUDA events around each call (median of 7 after 3
warm-ups); checks the labels are identical and that this build is faster.
Prints both timings (run with -s to see them).
"""

import statistics

import numpy as np
import pytest
import torch

import refmod
from dbscan_torch import dbscan2d, synthetic

pytestmark = pytest.mark.gpu


def _time(fn, X, reps=7, warm=3):
    for _ in range(warm):
        fn(X, 0.5, 10)
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        lab = fn(X, 0.5, 10)
        b.record()
        torch.cuda.synchronize()
        out.append(a.elapsed_time(b))
    return statistics.median(out), lab


def test_faster_than_reference_cuda_at_10m():
    ref = refmod.load("cuda")
    if ref is None:
        pytest.skip("reference CUDA build not present in oracle/_ref/cuda")
    X = torch.from_numpy(synthetic.constant_density(10_000_000, seed=0)).cuda()
    ours_ms, ours = _time(dbscan2d, X)
    ref_ms, want = _time(ref.dbscan2d, X)
    _, prof = ref.dbscan2d_profile(X, 0.5, 10)
    print(f"\n10M constant density: ours {ours_ms:.3f} ms ({10_000 / ours_ms:.1f} Mpts/s), "
          f"reference CUDA {ref_ms:.3f} ms ({10_000 / ref_ms:.1f} Mpts/s), "
          f"speed-up {ref_ms / ours_ms:.2f}x")
    print("reference CUDA stages (ms):", {k: round(v, 3) for k, v in sorted(prof.items())})
    assert np.array_equal(ours.cpu().numpy(), want.cpu().numpy())
    assert ours_ms < ref_ms
