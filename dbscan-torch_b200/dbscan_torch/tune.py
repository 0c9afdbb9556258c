"""Launch-shape autotuner for fixed-layout batched runs.

Six kernels of the pipeline walk their work with grid-stride loops or dynamic
work counters, so their grids (blocks per SM) can change without changing a
label: the per-key count of the counting sort, the cell pass (boxes,
neighbour rows, point classes), the core counts, the candidate-pair listing,
the pair tests with their unions, and the label pass. Their best grids depend
on the layout (cloud sizes, densities, how many clouds), which a
``BatchedPlan`` fixes; ``BatchedPlan.tune()`` times shapes on the plan's own
buffers with CUDA events and keeps the fastest.

The search is a coordinate descent: starting from the built-in shape, each
kernel in turn tries every candidate grid with the others held, and a move is
kept only when it beats the best time so far by more than ``min_gain`` (a
relative margin, so that timing noise does not pick a shape).
"""

from __future__ import annotations

from typing import Callable, Dict, Sequence, Tuple

TUNED = ("count", "cell_prep", "core", "pairs", "pair_scan", "labels")
CANDIDATES = (2, 4, 8, 16, 32)
MAX_BLOCKS_PER_SM = 32

Shape = Tuple[int, ...]


def coordinate_descent(measure: Callable[[Shape], float], start: Sequence[int],
                       candidates: Sequence[int] = CANDIDATES, rounds: int = 1,
                       min_gain: float = 0.01) -> Tuple[Shape, float, Dict[Shape, float]]:
    """Minimise ``measure(shape)`` (a time) one coordinate at a time.

    Returns the best shape, its time and every shape measured with its time.
    Each shape is measured once; ``rounds`` sweeps over the coordinates stop
    early when a sweep moves nothing.
    """
    if len(start) != len(TUNED):
        raise ValueError(f"a shape has {len(TUNED)} entries")
    for v in list(start) + list(candidates):
        if not 1 <= int(v) <= MAX_BLOCKS_PER_SM:
            raise ValueError(f"blocks per SM must be in [1, {MAX_BLOCKS_PER_SM}], got {v}")
    best = tuple(int(v) for v in start)
    trials: Dict[Shape, float] = {best: float(measure(best))}
    best_t = trials[best]
    for _ in range(rounds):
        moved = False
        for k in range(len(best)):
            for v in candidates:
                cand = best[:k] + (int(v),) + best[k + 1:]
                if cand not in trials:
                    trials[cand] = float(measure(cand))
                if trials[cand] < best_t * (1.0 - min_gain):
                    best, best_t, moved = cand, trials[cand], True
        if not moved:
            break
    return best, best_t, trials
