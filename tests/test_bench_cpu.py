"""bench.py's host-side contract, without a GPU: the reference arm imports
nothing of this build (only the generators, by file, and the reference's own
module), both arms describe the workload with the same config, and the CPU
baseline leg runs in a child process of its own and prints one JSON line."""

import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_loads_nothing_of_this_build():
    code = (
        "import sys\n"
        "sys.argv = ['bench.py']\n"
        "import bench\n"
        "X = bench._synthetic().constant_density(2000, seed=0)\n"
        "assert X.shape == (2000, 2)\n"
        "assert 'dbscan_torch' not in sys.modules, 'package imported'\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libdbscan_b200' not in maps and 'dbscan_torch/_C' not in maps, 'native code loaded'\n"
        "assert bench.base_config(1) == bench.base_config(1)\n"
    )
    subprocess.run([sys.executable, "-c", code], cwd=ROOT, check=True, timeout=300)


def test_cpu_leg_child_process(tmp_path):
    sys.path.insert(0, os.path.join(ROOT, "dbscan-torch_b200"))
    from dbscan_torch.synthetic import constant_density
    pts = tmp_path / "points.npy"
    np.save(pts, constant_density(20_000, seed=1))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--leg", "cpu",
                        "--points-file", str(pts)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
    base = json.loads(line)
    assert base["kind"] in ("reference", "port") and base["value"] > 0 and base["cores"] >= 1
    assert "fresh process" in base["sample"]
