"""Shared test setup: import paths, the `gpu` marker, small helpers.

Tests marked `gpu` need a CUDA device (run on a B200); everything else runs
on CPU: the oracle against golden vectors and the reference's own CPU path,
host-side validation, and the C-ABI library's exports.
"""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "dbscan-torch_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

# Device failures are checked synchronously after every call in tests.
os.environ.setdefault("DBSCAN_TORCH_SYNC", "1")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available() -> bool:
    import torch
    return torch.cuda.is_available()


def pytest_collection_modifyitems(config, items):
    if cuda_available():
        return
    skip = pytest.mark.skip(reason="CUDA not available")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def canonical(labels: np.ndarray) -> np.ndarray:
    """First-appearance relabelling (noise stays -1), as the reference tests'
    _relabel / _canonical (test_basic.py:23-39, test_eps_boundary.py:162-171)."""
    labels = np.asarray(labels)
    out = np.full(labels.shape, -1, dtype=np.int64)
    pos = labels >= 0
    if pos.any():
        _, first = np.unique(labels[pos], return_index=True)
        order = np.argsort(first)
        uniq = np.unique(labels[pos])[order]
        remap = {int(u): i for i, u in enumerate(uniq)}
        out[pos] = np.array([remap[int(v)] for v in labels[pos]])
    return out
