"""Serving loop: many independent clustering requests under a device-memory
budget, continuously batched into segmented pipeline runs.

No counterpart in the reference (it clusters one cloud per call). Each
request has the semantics of a plain ``dbscan2d`` call on its own cloud: its
labels are numbered from 0 and equal that call's labels bit for bit.

Structure:

* **Arena.** ``lanes`` (default 3) fixed sets of device buffers, allocated
  once: points, labels, per-cloud tables and one pipeline workspace, each set
  sized for ``lane_points`` points and ``lane_clouds`` clouds. The whole arena
  (``arena_bytes``) stays under ``budget_bytes``. Each lane has its own
  stream, so one batch's copies in, pipeline and copies out overlap with
  the other lanes' (three lanes keep the copy engines and the SMs busy at
  once; two lanes saturated about 15% lower on the serving benchmark).
* **Footprint and admission.** ``footprint_bytes(n)`` is what a request of n
  points occupies in a lane (workspace share plus points and labels). A
  request joins a batch while the batch's points and cloud count fit the lane;
  a request larger than a whole lane is refused at ``submit``.
* **Continuous batching.** ``step()`` retires finished batches and, whenever a
  lane is free and requests are queued, launches every queued request that
  fits (first come, first served) as one batched pipeline run, enqueued by
  one native call (``_C.serve_launch``): one host-to-device copy per request
  into the lane's point buffer, one copy of the cloud tables, the segmented
  pipeline, one device-to-host copy of the batch's labels into one pinned
  block of the server's host arena (each request's ``labels`` is a view of
  it, so the block returns to the arena with the batch's last result;
  ``clone()`` a result to keep it alone), and one of the device status word.
  The host arena is pinned once, at construction: pinning host memory while
  serving (a caching pinned allocator growing) stalled the loop for up to
  130 ms at a time. Completion is
  observed through CUDA events, never by blocking the host;
  ``pop_finished()`` hands back the requests completed since its last call.

Host inputs should be pinned (``torch.Tensor.pin_memory()``) for the copies
to be asynchronous.
"""

from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field
from typing import Deque, List, Optional

import torch

from . import _C


def footprint_bytes(n: int, nseg: int = 1) -> int:
    """Device bytes a batch of ``nseg`` clouds holding ``n`` points occupies:
    pipeline workspace, float32 (n, 2) points and int32 labels."""
    return int(_C.workspace_bytes(max(int(n), 1), max(int(nseg), 1))) + 12 * int(n) + 24 * int(nseg)


@dataclass
class Request:
    """One clustering request. ``labels`` (a pinned CPU int32 tensor) holds
    the result once ``done``; ``t_submit`` / ``t_done`` are
    ``time.perf_counter()`` stamps."""
    X: torch.Tensor
    eps: float
    min_samples: int
    t_submit: float
    rid: int
    labels: Optional[torch.Tensor] = None
    t_done: float = 0.0
    done: bool = False

    @property
    def n(self) -> int:
        return int(self.X.shape[0])

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


@dataclass
class _Lane:
    stream: torch.cuda.Stream
    X: torch.Tensor
    labels: torch.Tensor
    offsets: torch.Tensor
    params: torch.Tensor
    ws: torch.Tensor
    offsets_host: torch.Tensor
    params_host: torch.Tensor
    status_host: torch.Tensor
    event: torch.cuda.Event
    batch: List[Request] = field(default_factory=list)
    busy: bool = False


class DbscanServer:
    """Continuous-batching DBSCAN server on one device (see module docstring).

    Admission: the lanes are sized once from min(budget_bytes, free device
    memory - RESERVE_BYTES) (``torch.cuda.mem_get_info`` at construction);
    each lane holds a batch whose footprint (``footprint_bytes`` of its points
    and clouds) is at most the lane's. Because the lanes are the whole arena,
    admitting a request into a lane is admitting its footprint against the
    free-memory budget, without a device allocation per batch.

    Args:
        budget_bytes: device memory the arena may use (default 64 GiB).
        lane_points: points per lane; default: the largest that keeps the
            arena under the budget, capped at 64M points.
        lane_clouds: clouds per lane (per batch).
        lanes: number of lanes (concurrent batches).
        host_arena_bytes: pinned host memory for the served labels, pinned
            once here (default: twice the labels of all lanes, at most
            512 MiB; 0 takes every batch's label block from torch's caching
            pinned allocator instead, which pins new blocks while serving).
    """

    RESERVE_BYTES = 1 << 30  # free memory left to the caller

    def __init__(self, budget_bytes: int = 64 << 30, lane_points: Optional[int] = None,
                 lane_clouds: int = 1024, lanes: int = 3, device=None,
                 host_arena_bytes: Optional[int] = None):
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        if lanes < 1 or lane_clouds < 1:
            raise ValueError("lanes and lane_clouds must be >= 1")
        # The arena is carved once, from the budget or the free device memory
        # at construction (less a reserve for the caller's own tensors),
        # whichever is smaller.
        free, _ = torch.cuda.mem_get_info(self.device)
        self.free_bytes_at_start = int(free)
        usable = min(int(budget_bytes), max(0, int(free) - self.RESERVE_BYTES))
        per_lane = usable // lanes
        if lane_points is None:
            lo, hi = 1, 64 << 20
            while lo < hi:  # largest lane_points whose footprint fits per_lane
                mid = (lo + hi + 1) // 2
                if footprint_bytes(mid, lane_clouds) <= per_lane:
                    lo = mid
                else:
                    hi = mid - 1
            lane_points = lo
        if footprint_bytes(lane_points, lane_clouds) > per_lane:
            raise ValueError(f"a lane of {lane_points} points and {lane_clouds} clouds needs "
                             f"{footprint_bytes(lane_points, lane_clouds)} bytes, more than "
                             f"min(budget_bytes, free device memory - reserve) / lanes = {per_lane}")
        self.budget_bytes = int(budget_bytes)
        self.lane_points = int(lane_points)
        self.lane_clouds = int(lane_clouds)
        self.arena_bytes = lanes * footprint_bytes(lane_points, lane_clouds)
        self.lanes: List[_Lane] = []
        for _ in range(lanes):
            P, S, d = self.lane_points, self.lane_clouds, self.device
            self.lanes.append(_Lane(
                stream=torch.cuda.Stream(device=d),
                X=torch.zeros((P, 2), dtype=torch.float32, device=d),
                labels=torch.empty(P, dtype=torch.int32, device=d),
                offsets=torch.zeros(S + 1, dtype=torch.int64, device=d),
                params=torch.zeros(S * 16, dtype=torch.uint8, device=d),
                ws=torch.empty(int(_C.workspace_bytes(P, S)), dtype=torch.uint8, device=d),
                offsets_host=torch.zeros(S + 1, dtype=torch.int64).pin_memory(),
                params_host=torch.zeros(S * 16, dtype=torch.uint8).pin_memory(),
                status_host=torch.zeros(4, dtype=torch.uint8).pin_memory(),
                event=torch.cuda.Event(),
            ))
        if host_arena_bytes is None:
            host_arena_bytes = min(2 * lanes * self.lane_points * 4, 512 << 20)
        self.host_arena = _C.PinnedArena(int(host_arena_bytes)) if host_arena_bytes > 0 else None
        self.queue: Deque[Request] = collections.deque()
        self._next_id = 0
        self.batches = 0
        self.completed = 0
        self._finished: List[Request] = []
        self._track_finished = False  # set by the first pop_finished() call

    # ------------------------------------------------------------- requests
    def submit(self, X: torch.Tensor, eps: float, min_samples: int, t_submit: Optional[float] = None) -> Request:
        """Queue one cloud (float32 (N, 2) CPU tensor, ideally pinned)."""
        if X.dim() != 2 or X.size(1) != 2:
            raise RuntimeError("X must have shape (N, 2)")
        if X.dtype != torch.float32:
            raise RuntimeError("X must be float32")
        if not eps > 0:
            raise RuntimeError("eps must be > 0")
        if min_samples < 1:
            raise RuntimeError("min_samples must be >= 1")
        if X.size(0) > self.lane_points:
            raise RuntimeError(f"request of {X.size(0)} points exceeds the lane capacity of "
                               f"{self.lane_points} points (budget {self.budget_bytes} bytes)")
        r = Request(X=X.contiguous(), eps=float(eps), min_samples=int(min_samples),
                    t_submit=time.perf_counter() if t_submit is None else t_submit, rid=self._next_id)
        self._next_id += 1
        self.queue.append(r)
        return r

    # ----------------------------------------------------------------- loop
    def step(self) -> int:
        """Retire finished batches, launch new ones on free lanes. Returns the
        number of requests completed by this call. Never blocks on the GPU."""
        done = 0
        for lane in self.lanes:
            if lane.busy and lane.event.query():
                done += self._retire(lane)
        for lane in self.lanes:
            if not lane.busy and self.queue:
                self._launch(lane)
        return done

    def pop_finished(self) -> List[Request]:
        """The requests completed since the last call, in completion order
        (a caller holding many requests in flight need not scan them all for
        ``done``). Requests are collected from the first call on, so a
        caller that never calls it keeps nothing alive here."""
        self._track_finished = True
        out, self._finished = self._finished, []
        return out

    def drain(self) -> None:
        """Run until every submitted request is done."""
        while self.queue or any(l.busy for l in self.lanes):
            if self.step() == 0:
                time.sleep(20e-6)

    def _launch(self, lane: _Lane) -> None:
        batch: List[Request] = []
        total = 0
        while self.queue and len(batch) < self.lane_clouds and total + self.queue[0].n <= self.lane_points:
            r = self.queue.popleft()
            batch.append(r)
            total += r.n
        if not batch:
            return
        with torch.cuda.stream(lane.stream):
            # One call enqueues the whole batch on the lane's stream: the
            # cloud tables, one copy in per request, the segmented pipeline,
            # one copy out per request into its own pinned label tensor, the
            # status word. The previous batch of this lane has retired, so
            # its pinned staging tensors can be rewritten.
            labels = _C.serve_launch([r.X for r in batch], [r.eps for r in batch],
                                     [r.min_samples for r in batch], lane.X, lane.offsets_host, lane.offsets,
                                     lane.params_host, lane.params, lane.labels, lane.ws, lane.status_host,
                                     self.host_arena)
            lane.event.record(lane.stream)
        for r, lab in zip(batch, labels):
            r.labels = lab
        lane.batch = batch
        lane.busy = True
        self.batches += 1

    def _retire(self, lane: _Lane) -> int:
        st = int(lane.status_host.view(torch.int32)[0]) if lane.batch and sum(r.n for r in lane.batch) else 0
        if st:
            raise RuntimeError(f"dbscan2d (serving): device-side failure (status 0x{st:x}) in a batch of "
                               f"{len(lane.batch)} requests; their labels are invalid")
        now = time.perf_counter()
        for r in lane.batch:
            r.t_done = now
            r.done = True
        if self._track_finished:
            self._finished.extend(lane.batch)
        n = len(lane.batch)
        self.completed += n
        lane.batch = []
        lane.busy = False
        return n
