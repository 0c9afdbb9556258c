"""Generate golden fixtures from the reference's own CUDA build.

Runs ryanirl/dbscan-torch's CUDA path (built from its sources by
oracle/build_ref.py into oracle/_ref/cuda) on small seeded inputs and stores,
per case, the input, eps, min_samples, the labels and the per-stage
intermediates of its debug entry point (dbscan_cuda.cu:777-789). Needs a GPU;
run it on a B200, then copy the .npz files from OUTDIR next to this script:

    python tests/golden/make_golden.py --out OUTDIR

tests/test_oracle.py checks the CPU oracle against every fixture bit for bit.
"""

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")]

import datasets  # noqa: E402
import probes  # noqa: E402
import refmod  # noqa: E402

KEEP = {"three_blobs", "three_blobs_eps06", "uniform_ms1", "lattice_exact_eps_ms5", "spirals",
        "dense_square_ms4", "offset_negative", "tiny_eps", "single_point_ms1", "all_noise",
        "duplicates", "wide_sparse", "moons_1k", "circles_2k"}


def cases():
    rng = np.random.default_rng(99)
    out = [(n, X, e, m) for n, X, e, m in datasets.parity_cases() if n in KEEP]
    out.append(("dense_blobs_8k", datasets.dense_overlapping_blobs(8000, 3), 0.5, 5))
    out.append(("uniform_8k", datasets.near_percolation_uniform(8000, 5), 0.5, 5))
    for fam, fn in probes.FAMILIES.items():
        X, eps, ms, _, _ = fn(count=600, seed=11)
        out.append((f"probe_{fam}", X, eps, ms))
    out.append(("straddle_zero", rng.normal(0, 3.0, size=(6000, 2)).astype(np.float32), 0.4, 4))
    return out


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    ref = refmod.load("cuda")
    if ref is None or not torch.cuda.is_available():
        print("needs the reference CUDA build and a GPU")
        return 1
    os.makedirs(a.out, exist_ok=True)
    names = ["labels", "keys_sorted", "perm", "xs", "ys", "is_core", "cell_start",
             "cluster_id_per_cell", "uf", "sorted_labels_pre_border", "sorted_labels_final"]
    for name, X, eps, ms in cases():
        outs = ref.dbscan2d_cuda_debug(torch.from_numpy(X).cuda(), eps, ms)
        rec = {k: t.cpu().numpy() for k, t in zip(names, outs)}
        lab = ref.dbscan2d(torch.from_numpy(X).cuda(), eps, ms).cpu().numpy()
        assert np.array_equal(lab, rec["labels"])
        np.savez_compressed(os.path.join(a.out, f"{name}.npz"), X=X, eps=np.float64(eps),
                            min_samples=np.int64(ms), labels=rec["labels"], perm=rec["perm"],
                            is_core=rec["is_core"], cell_start=rec["cell_start"],
                            cluster_id_per_cell=rec["cluster_id_per_cell"], uf=rec["uf"],
                            sorted_labels_pre_border=rec["sorted_labels_pre_border"],
                            sorted_labels_final=rec["sorted_labels_final"])
        print(f"{name}: n={X.shape[0]} clusters={int(lab.max()) + 1} noise={int((lab < 0).sum())}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
