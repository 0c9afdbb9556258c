"""dbscan_torch (B200 build): grid-hashed 2D DBSCAN on hand-written sm_100a kernels.

Drop-in for the Python surface of ryanirl/dbscan-torch v0.2.0
(dbscan_torch/__init__.py:57-119): the functional ``dbscan2d`` and the
sklearn-style ``DBSCAN`` class keep their names, arguments, return types and
error messages. Labels are bit-identical to the reference's CUDA path,
cluster numbering included.

Differences from the reference, by design of this build:
  * every call runs on a CUDA device; a CPU tensor (or numpy array through
    ``DBSCAN``) is copied to the current CUDA device and the labels copied
    back, and a machine without a GPU gets a RuntimeError (the reference ran
    a separate CPU implementation for CPU tensors);
  * ``dbscan2d_batched`` clusters many clouds, each with its own eps and
    min_samples, in one pipeline run (see also ``BatchedPlan`` for a
    CUDA-graph-captured batch and ``dbscan_torch.serving`` for continuous
    batching of a request stream).
"""

from __future__ import annotations

from importlib.metadata import PackageNotFoundError
from importlib.metadata import version as _pkg_version
from typing import Any, Optional, Sequence, Union

import numpy as np
import torch

try:
    from ._build_info import BUILD_TORCH_VERSION as _build_torch
except ImportError:
    _build_torch = None

if _build_torch is not None:
    # Same guard as the reference (dbscan_torch/__init__.py:17-38): the C++
    # extension only loads against the torch minor version it was built for.
    try:
        _mismatch = tuple(int(x) for x in _build_torch.split(".")[:2]) != tuple(
            int(x) for x in torch.__version__.split(".")[:2])
    except (ValueError, IndexError, AttributeError):
        _mismatch = False
    if _mismatch:
        raise ImportError(
            f"dbscan_torch was built against torch {_build_torch} but the installed "
            f"runtime torch is {torch.__version__}. Rebuild with "
            f"`python dbscan-torch_b200/build.py --force`.")

try:
    from . import _C
except ImportError as e:  # pragma: no cover - exercised only on a broken build
    raise ImportError(
        "dbscan_torch: the native extension (_C + libdbscan_b200.so) is missing or "
        "failed to load; build it with `python dbscan-torch_b200/build.py`. "
        f"Loader error: {e}") from e

ArrayLike2D = Union[np.ndarray, torch.Tensor]

__all__ = [
    "dbscan2d", "dbscan2d_profile", "dbscan2d_batched", "DBSCAN", "ArrayLike2D",
    "BatchedPlan", "DbscanServer", "footprint_bytes", "shard_clouds", "check_status",
]

try:
    __version__ = _pkg_version("dbscan-torch")
except PackageNotFoundError:
    __version__ = "0.2.0+b200"


def dbscan2d(X: torch.Tensor, eps: float, min_samples: int) -> torch.Tensor:
    """Run DBSCAN on a 2D point set.

    Args:
        X: float32 tensor of shape (N, 2).
        eps: neighborhood radius (> 0).
        min_samples: minimum neighbors (incl. self) to be a core point (>= 1).

    Returns:
        int32 tensor of shape (N,) on X's device. -1 indicates noise, otherwise
        a cluster id in ``[0, n_clusters)``.
    """
    return _C.dbscan2d(X, float(eps), int(min_samples))


def dbscan2d_profile(X: torch.Tensor, eps: float, min_samples: int):
    """Labels plus ``{stage_name: ms}`` GPU time per reference stage."""
    return _C.dbscan2d_profile(X, float(eps), int(min_samples))


def _as_cpu(v, dtype) -> torch.Tensor:
    if isinstance(v, torch.Tensor):
        return v.detach().to("cpu", dtype)
    return torch.as_tensor(np.asarray(v), dtype=dtype)


def dbscan2d_batched(X: torch.Tensor, seg_offsets: Sequence[int], eps, min_samples) -> torch.Tensor:
    """Cluster many clouds in one pipeline run.

    Clouds are concatenated in ``X``: cloud ``s`` owns rows
    ``seg_offsets[s]:seg_offsets[s+1]`` and uses ``eps[s]`` and
    ``min_samples[s]`` (scalars are broadcast). The labels of each cloud are
    numbered from 0 and equal ``dbscan2d`` on that cloud alone.
    """
    off = _as_cpu(seg_offsets, torch.int64)
    S = off.numel() - 1
    ep = _as_cpu(eps, torch.float64).reshape(-1)
    ms = _as_cpu(min_samples, torch.int64).reshape(-1)
    if ep.numel() == 1 and S > 1:
        ep = ep.expand(S).contiguous()
    if ms.numel() == 1 and S > 1:
        ms = ms.expand(S).contiguous()
    return _C.dbscan2d_batched(X, off, ep, ms)


def check_status() -> None:
    """Wait for every pending call; raise RuntimeError if one recorded a
    device-side failure (a bounded wait that ran out)."""
    _C.check_status()


class DBSCAN:
    """sklearn-compatible class wrapper around :func:`dbscan2d`.

    Mirrors the reference's class (dbscan_torch/__init__.py:76-119): numpy in
    -> numpy out, torch in -> torch out on the same device, non-float32 input
    is cast, ``fit`` returns self, ``y`` is ignored.
    """

    def __init__(self, eps: float = 0.5, min_samples: int = 5):
        self.eps = float(eps)
        self.min_samples = int(min_samples)
        self.labels_: Optional[ArrayLike2D] = None

    def fit(self, X: ArrayLike2D, y: Any = None) -> "DBSCAN":
        is_torch = isinstance(X, torch.Tensor)
        if is_torch:
            Xt = X if X.dtype == torch.float32 else X.to(torch.float32)
        else:
            Xt = torch.as_tensor(X, dtype=torch.float32)
        labels = dbscan2d(Xt, self.eps, self.min_samples)
        self.labels_ = labels if is_torch else labels.cpu().numpy()
        return self

    def fit_predict(self, X: ArrayLike2D, y: Any = None) -> ArrayLike2D:
        return self.fit(X, y).labels_  # type: ignore[return-value]


from .batched import BatchedPlan  # noqa: E402  (needs _C)
from .serve import DbscanServer, footprint_bytes  # noqa: E402  (needs _C)
from .shard import shard_clouds  # noqa: E402
