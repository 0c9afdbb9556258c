"""Inputs on which the arithmetic forms of the squared-distance test disagree.

The reference build compiles `ex*ex + ey*ey` with --use_fast_math
(setup.py:77-83), so nvcc may contract it into a fused multiply-add, and
which product it fuses is not visible in the source. Three candidate forms:
unfused, fma(ex, ex, ey*ey) and fma(ey, ey, ex*ex). These families place
point pairs at float32 distances within an ulp of eps where the forms give
different verdicts, one pair per isolated slot, and read the verdicts of one
group of call sites from the labels:

  unite   two coincident min_samples-groups (both core wholesale): merged
          iff box_box_d2, point_box_d2 and the pair test in k_unite_pairs
          (dbscan_cuda.cu:351, 359, 363) all accept;
  core    two single points with min_samples 2: core iff point_box_d2 and
          the pair test in k_core_pass2 (:235, :239) accept;
  border  a non-core point next to a core point whose other neighbours sit
          on the far side: border iff point_box_d2 and the pair test in
          k_border_assign (:453, :458) accept.
"""

from __future__ import annotations

import numpy as np

import oracle

EPS = 1.0
SPACING = 4.0


def _step(v: np.ndarray, k: int) -> np.ndarray:
    out = v.copy()
    d = np.float32(np.inf) if k > 0 else np.float32(-np.inf)
    for _ in range(abs(k)):
        out = np.nextafter(out, d)
    return out


def borderline_pairs(count: int, seed: int):
    """Returns (P, Q, verdicts) with verdicts[k] = (unfused, fma_x, fma_y)
    acceptances of |Q - P| <= EPS, not all equal for any k."""
    rng = np.random.default_rng(seed)
    side = int(np.ceil(np.sqrt(count)))
    k = np.arange(count)
    base = np.stack([(k % side) * SPACING, (k // side) * SPACING], 1) - SPACING * side / 2
    P = (base + rng.uniform(-0.5, 0.5, size=(count, 2))).astype(np.float32)
    chosen_q = np.zeros((count, 2), np.float32)
    verdict = np.zeros((count, 3), bool)
    found = np.zeros(count, bool)
    for _attempt in range(24):
        todo = np.flatnonzero(~found)
        if todo.size == 0:
            break
        th = rng.uniform(0, 2 * np.pi, size=todo.size)
        q0 = (P[todo].astype(np.float64) + EPS * np.stack([np.cos(th), np.sin(th)], 1)).astype(np.float32)
        for i in range(-4, 5):
            for j in range(-4, 5):
                sel = todo[~found[todo]]
                if sel.size == 0:
                    break
                pos = np.searchsorted(todo, sel)
                q = np.stack([_step(q0[pos, 0], i), _step(q0[pos, 1], j)], 1)
                v = np.stack([oracle.pair_d2_batch(P[sel], q, f) <= np.float32(EPS * EPS)
                              for f in (oracle.FORM_UNFUSED, oracle.FORM_FMA_X, oracle.FORM_FMA_Y)], 1)
                hit = v.any(1) & ~v.all(1)
                chosen_q[sel[hit]] = q[hit]
                verdict[sel[hit]] = v[hit]
                found[sel[hit]] = True
    keep = np.flatnonzero(found)
    return P[keep], chosen_q[keep], verdict[keep]


def family_unite(count=2048, seed=0, group=2):
    P, Q, v = borderline_pairs(count, seed)
    X = np.concatenate([np.repeat(P, group, 0), np.repeat(Q, group, 0)]).astype(np.float32)
    slot = np.concatenate([np.repeat(np.arange(len(P)), group), np.repeat(np.arange(len(P)), group)])
    return X, EPS, group, slot, v


def family_core(count=2048, seed=1):
    P, Q, v = borderline_pairs(count, seed)
    X = np.concatenate([P, Q]).astype(np.float32)
    slot = np.concatenate([np.arange(len(P)), np.arange(len(P))])
    return X, EPS, 2, slot, v


def family_border(count=2048, seed=2):
    B, Q, v = borderline_pairs(count, seed)
    s = np.sign(Q - B).astype(np.float32)
    s[s == 0] = 1
    R1 = (Q + np.float32(0.30) * s).astype(np.float32)
    R2 = (Q + np.float32(0.35) * s).astype(np.float32)
    X = np.concatenate([B, Q, R1, R2]).astype(np.float32)
    n = len(B)
    slot = np.concatenate([np.arange(n)] * 4)
    return X, EPS, 3, slot, v


FAMILIES = {"unite": family_unite, "core": family_core, "border": family_border}
SITES_OF = {"unite": (2, 3, 4), "core": (0, 1), "border": (5, 6)}


def slot_signature(labels: np.ndarray, slot: np.ndarray) -> np.ndarray:
    """Per slot, a code of how its points are labelled: the canonical label
    pattern in point order (noise -1, else first-appearance ids)."""
    order = np.lexsort((np.arange(len(slot)), slot))
    lab = labels[order]
    sl = slot[order]
    nslot = sl.max() + 1 if sl.size else 0
    counts = np.bincount(sl, minlength=nslot)
    width = counts.max() if counts.size else 0
    sig = np.full((nslot, width), -2, np.int64)
    start = np.concatenate([[0], np.cumsum(counts)])
    for s in range(nslot):
        seg = lab[start[s]:start[s + 1]]
        seen = {}
        for t, x in enumerate(seg):
            if x < 0:
                sig[s, t] = -1
            else:
                sig[s, t] = seen.setdefault(int(x), len(seen))
    return sig
