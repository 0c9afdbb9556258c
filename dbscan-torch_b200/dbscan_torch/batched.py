"""Batched DBSCAN on device-resident buffers, optionally replayed as a CUDA graph.

``dbscan2d_batched`` (package root) takes host-side cloud tables and runs one
pipeline over all clouds. ``BatchedPlan`` keeps every buffer on the device
for a fixed layout (cloud sizes) so that the whole pipeline -- about twenty
kernel launches with no host synchronisation -- is captured once in a CUDA
graph and replayed for each new batch of points / parameters.
``BatchedPlan.tune()`` picks the grids of the pipeline's grid-stride kernels
for the plan's layout (see ``tune.py``).
"""

from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch

from . import _C
from . import tune as _tune


class BatchedPlan:
    """Fixed-layout batch: ``len(seg_offsets) - 1`` clouds, cloud ``s`` in rows
    ``seg_offsets[s]:seg_offsets[s+1]`` of the point buffer.

    ``run(X, eps, min_samples)`` copies the inputs into the plan's buffers,
    launches (or replays) the pipeline on the current stream and returns the
    plan's label buffer (valid until the next ``run``).
    """

    def __init__(self, seg_offsets: Sequence[int], device=None, use_graph: bool = True):
        off = torch.as_tensor(np.asarray(seg_offsets, dtype=np.int64))
        if off.dim() != 1 or off.numel() < 2 or int(off[0]) != 0:
            raise ValueError("seg_offsets must be a 1-D sequence starting at 0 with >= 2 entries")
        if bool((off[1:] < off[:-1]).any()):
            raise ValueError("seg_offsets must be non-decreasing")
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self.nseg = off.numel() - 1
        self.n = int(off[-1])
        self.seg_offsets_host = off
        self.seg_offsets = off.to(self.device)
        self.X = torch.zeros((self.n, 2), dtype=torch.float32, device=self.device)
        self.labels = torch.full((self.n,), -1, dtype=torch.int32, device=self.device)
        self.params = torch.zeros(self.nseg * 16, dtype=torch.uint8, device=self.device)
        self.ws = torch.empty(_C.workspace_bytes(max(self.n, 1), self.nseg), dtype=torch.uint8,
                              device=self.device)
        self._params_host = torch.zeros(self.nseg * 16, dtype=torch.uint8).pin_memory()
        self.use_graph = use_graph
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        self.shape: Optional[tuple] = None  # None = built-in launch shape

    def set_params(self, eps, min_samples) -> None:
        ep = torch.as_tensor(np.broadcast_to(np.asarray(eps, dtype=np.float64), (self.nseg,)).copy())
        ms = torch.as_tensor(np.broadcast_to(np.asarray(min_samples, dtype=np.int64), (self.nseg,)).copy())
        self._params_host.copy_(_C.fill_seg_params(ep, ms))
        self.params.copy_(self._params_host, non_blocking=True)

    def _launch(self, shape=None) -> None:
        shape = self.shape if shape is None else shape
        _C.dbscan2d_batched_into(self.X, self.seg_offsets, self.params, self.labels, self.ws,
                                 list(shape) if shape is not None else [])

    def set_shape(self, shape) -> None:
        """Launch shape for later runs: blocks per SM of the tuned kernels
        (``tune.TUNED`` order; 0 = built-in), or None for the built-in shape.
        A captured graph is dropped and captured again at the next run."""
        if shape is not None:
            shape = tuple(int(v) for v in shape)
            if len(shape) != len(_tune.TUNED) or not all(0 <= v <= _tune.MAX_BLOCKS_PER_SM for v in shape):
                raise ValueError(f"shape must hold {len(_tune.TUNED)} entries in [0, {_tune.MAX_BLOCKS_PER_SM}]")
        self.shape = shape
        self.graph = None

    def tune(self, reps: int = 3, candidates: Sequence[int] = _tune.CANDIDATES, rounds: int = 1,
             min_gain: float = 0.01) -> dict:
        """Time launch shapes on the plan's current points and parameters
        (eager launches on the current stream, CUDA events, best of ``reps``
        runs per shape), keep the fastest for later runs and return
        ``{"shape", "ms", "default_shape", "default_ms", "trials"}``. Labels
        do not depend on the shape; the plan's labels afterwards are those of
        the last shape timed."""
        default = tuple(int(v) for v in _C.default_launch_shape(self.n))
        if self.n == 0:
            return {"shape": default, "ms": 0.0, "default_shape": default, "default_ms": 0.0, "trials": 0}
        stream = torch.cuda.current_stream(self.device)

        def measure(shape):
            best = float("inf")
            for _ in range(max(1, reps)):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                self._launch(shape)
                b.record(stream)
                b.synchronize()
                best = min(best, a.elapsed_time(b))
            return best

        start = self.shape if self.shape is not None and all(self.shape) else default
        shape, t, trials = _tune.coordinate_descent(measure, start, candidates, rounds, min_gain)
        st = self.status()
        if st != 0:
            raise RuntimeError(f"dbscan2d_batched: device status {st:#x} while tuning")
        self.set_shape(shape)
        return {"shape": shape, "ms": t, "default_shape": default, "default_ms": trials.get(default, float("nan")),
                "trials": len(trials)}

    def run(self, X: Optional[torch.Tensor] = None, eps=None, min_samples=None) -> torch.Tensor:
        if X is not None:
            if tuple(X.shape) != (self.n, 2):
                raise ValueError(f"X must have shape ({self.n}, 2)")
            self.X.copy_(X, non_blocking=True)
        if eps is not None or min_samples is not None:
            if eps is None or min_samples is None:
                raise ValueError("eps and min_samples go together")
            self.set_params(eps, min_samples)
        if self.n == 0:
            return self.labels
        if not self.use_graph:
            self._launch()
            return self.labels
        if self.graph is None:
            # One eager run initialises lazy state (kernel attributes) before
            # capture, on a side stream as torch's graph capture requires.
            side = torch.cuda.Stream(device=self.device)
            side.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(side):
                self._launch()
            torch.cuda.current_stream(self.device).wait_stream(side)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._launch()
            self.graph = g
        self.graph.replay()
        return self.labels

    def stats(self) -> dict:
        """Work counts of the last run (cells, sort form, hot-key slots, core
        queries, border points, union-find pairs); synchronises."""
        return dict(_C.read_stats(self.ws))

    def status(self) -> int:
        """Device status word of the last run (0 = ok); synchronises."""
        return int(_C.read_status(self.ws))
