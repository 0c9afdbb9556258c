"""Kernel launches of one dbscan2d call, counted with the profiler: the
figure bench.py reports as gpu_launches per step, and proof that the call
runs this library's kernels (names in namespace dbs::) and nothing else."""

import importlib.util
import os

import pytest
import torch

from dbscan_torch import dbscan2d, synthetic

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _kernels_of_one_call(X, eps, ms):
    dbscan2d(X, eps, ms)
    torch.cuda.synchronize()
    with torch.profiler.profile(activities=[torch.profiler.ProfilerActivity.CUDA]) as prof:
        dbscan2d(X, eps, ms)
        torch.cuda.synchronize()
    names = [e.name for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA]
    return [n for n in names if "k_" in n or "dbs::" in n], names


@pytest.mark.parametrize("kind", ["dense", "radix"])
def test_launches_per_call(kind):
    if kind == "dense":
        X = torch.from_numpy(synthetic.constant_density(200_000, seed=3)).cuda()
    else:
        # Two far-apart blobs: the key range is too sparse for the dense map,
        # so the radix sort runs.
        Xn = synthetic.blobs_with_noise(50_000, seed=4, n_blobs=2, noise_frac=0.0)
        Xn[: len(Xn) // 2] += 1.0e5
        X = torch.from_numpy(Xn).cuda()
    ours, names = _kernels_of_one_call(X, 0.5, 10)
    assert len(ours) == _bench().KERNELS_PER_CALL, names
    assert all("dbs::" in n for n in ours), names
    # Besides copies (the status read-back), the call launches nothing else.
    others = [n for n in names if not n.startswith(("Memcpy", "Memset"))]
    assert others == ours, names
