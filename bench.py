"""Benchmark of the dbscan2d hot path on B200 (one JSON line on stdout).

Workload: the constant-density cloud at N = 10,000,000 float32 points
(K = N/5,000 Gaussian blobs, sigma 1, centres uniform in a square of side
2*sqrt(N)/10, plus 2% uniform noise; eps 0.5, min_samples 10), seeded
synthetic data. One step = one dbscan2d call over the whole cloud.

  value     Mpoints/s of the pipeline with X resident in HBM (CUDA events on
            the launching stream around each call; L2 flushed between steps
            by writing a 512 MB buffer outside the timed events)
  e2e       same metric through the public API with HOST buffers: a pinned
            CPU tensor in, CPU labels out (H2D of X and D2H of labels inside
            the timed region)
  roofline  dominant stage: algorithmic bytes per launch / its average launch
            time (per-stage CUDA events of dbscan2d_profile), against the
            measured HBM copy bandwidth in MEASURED_PEAKS.json
  cpu_baseline    the reference's own CPU implementation (built from its
            sources into oracle/_ref/cpu) on the box's host cores, timed on
            the same workload in a fresh child process before this process
            touches the GPU
  reference_cuda  the reference's own CUDA implementation (oracle/_ref/cuda)
            on the same GPU and workload, in a child process run before this
            process touches the GPU: same warm-up, L2 flush and CUDA events,
            its per-stage split (dbscan2d_profile), and whether its labels
            equal this build's
  configs   the other plain-call workloads on the device: 100k blobs with
            noise, constant density at 1M and 5M, the adversarial 4M cloud
            (min_samples 4 and 32) (--no-configs skips them)
  batched   4,096 clouds (sizes log-uniform in [256, 262144]) in one batched
            pipeline run vs a loop of plain calls: clouds/s of each
            (--batched-clouds; 0 skips)
  serving   the Poisson request stream (2,000 req/s, sizes log-uniform in
            [1e3, 2e6], 60 s by default) through the continuous-batching
            server and through sequential plain calls: p50/p99 latency and
            clouds/s; then, for both, the highest offered rate whose p99 stays
            within 50 ms (--serve-seconds; 0 skips)

--impl reference times only the reference CPU path and prints its line (it
imports nothing of this build). Multi-GPU (torchrun): replicas only -- every
rank clusters its own cloud; the time is the max over ranks.
"""

from __future__ import annotations

import argparse
import gc
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "dbscan-torch_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "Mpoints/s @10M"
UNIT = "Mpoints/s"
N_POINTS = 10_000_000
EPS, MIN_SAMPLES = 0.5, 10
WORKLOAD = "constant_density_10M"
GENERATOR = "constant_density"
DATA = "synthetic (seeded constant-density Gaussian blobs + 2% noise)"
L2_FLUSH_BYTES = 512 << 20
# Kernel launches of one dbscan2d call (tests/test_launch_count.py counts them
# with the profiler): init, bounds, seg_finalize | csort_clear, csort_count,
# csort, keys, radix | rle | cell_prep, huge_bbox | core, status |
# 2 x (pairs, pair_scan, pair_warp) + flatten | ids, cid | labels. Kernels
# whose work the device-side plan skips (the sort form that does not run,
# the huge-cell pass without huge cells) still launch and return at once.
KERNELS_PER_CALL = 23
# Launches per reference stage (the profile entry point times stages).
STAGE_LAUNCHES = {"cell_keys": 3, "sort_gather": 5, "boundary_scan": 1, "build_ngh": 2,
                  "core_mark": 2, "union_find": 7, "cluster_id": 2, "border_assign": 1}
# The kernels that do a stage's work on this workload (the others of the
# stage return at once); the sort's depend on the form that ran.
SORT_KERNELS = {0: ("k_keys", "k_radix"), 1: ("k_csort_clear", "k_csort_count", "k_csort")}
SORT_FORM_NAME = {0: "radix", 1: "counting"}
STAGE_KERNEL = {"build_ngh": ("k_cell_prep",), "core_mark": ("k_core",),
                "border_assign": ("k_labels",)}
PROFILE_MD = os.path.join(ROOT, "profiles", "kernels_constant_density_10M.md")


def _synthetic():
    """The seeded generators (dbscan_torch/synthetic.py), loaded from their
    file so that nothing of the package -- in particular its native
    extension -- is imported (the reference arm must load the reference
    only)."""
    mod = sys.modules.get("dbs_bench_synthetic")
    if mod is None:
        path = os.path.join(PKG_DIR, "dbscan_torch", "synthetic.py")
        spec = importlib.util.spec_from_file_location("dbs_bench_synthetic", path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules["dbs_bench_synthetic"] = mod
    return mod


def _package():
    if PKG_DIR not in sys.path:
        sys.path.insert(0, PKG_DIR)
    import dbscan_torch
    return dbscan_torch


def base_config(world: int) -> dict:
    """The workload, identical in both arms' lines."""
    return {"workload": WORKLOAD, "n_points": N_POINTS, "eps": EPS, "min_samples": MIN_SAMPLES,
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (80 MB points, 40 MB labels, ~3.4 GB of pipeline arrays); "
                  "the GPU arm also writes a 512 MB buffer between timed steps, outside the events"}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region:
    one `nvidia-smi -lms 5` child started (and its first sample awaited)
    before timing begins, writing timestamped lines to a file -- no process
    is forked while the timed steps run -- and stopped afterwards (by its own
    PID). Only the samples stamped inside the timed window are summarised
    (the nearest ones when the window is shorter than the sampling period)."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._proc = None
        self._file = None

    def __enter__(self):
        self._file = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "5"],
                stdout=self._file, stderr=subprocess.DEVNULL)
            t_end = time.time() + 3.0
            while time.time() < t_end and os.path.getsize(self._file.name) == 0:
                time.sleep(0.02)
        except Exception:
            self._proc = None
        self._t0 = time.time()
        return self

    def __exit__(self, *a):
        self._t1 = time.time()
        if self._proc is not None:
            time.sleep(0.05)  # the samples of the last timed steps
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
        import datetime
        rows = []
        try:
            with open(self._file.name) as f:
                for line in f:
                    v = [x.strip() for x in line.split(",")]
                    if len(v) < 8:
                        continue
                    try:
                        ts = datetime.datetime.strptime(v[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                    except ValueError:
                        ts = None
                    rows.append((ts, v[1:]))
            os.unlink(self._file.name)
        except Exception:
            pass
        inside = [r for t, r in rows if t is not None and self._t0 <= t <= self._t1]
        if not inside and rows:  # window shorter than the sampling period
            mid = (self._t0 + self._t1) / 2
            timed = [(abs(t - mid), r) for t, r in rows if t is not None]
            inside = [min(timed, key=lambda x: x[0])[1]] if timed else [rows[-1][1]]
        self.samples = inside

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if len(s) > 3 + k and s[3 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def stage_bytes(n: int, cells: int, passes: int, kb: int) -> dict:
    """Algorithmic (compulsory) bytes per stage: each array the stage must
    touch, counted once (per-point and per-cell figures). passes == 0 means the
    counting sort over the dense key space ran (no radix passes)."""
    if passes == 0:
        # read X; write perm and the sorted float2 coordinates; cell_start,
        # cell_key, cell_seg per cell
        sort = n * (8 + 4 + 8) + cells * (4 + 8 + 4)
    else:
        # key + index read and written per pass, X gather, xy write
        sort = n * (passes * (2 * kb + 8) - 4 + 16)
    return {
        "cell_keys": n * 8,                                          # read X (bounds)
        "sort_gather": sort,
        "boundary_scan": 0 if passes == 0 else n * kb + cells * 16,  # sorted keys; cells
        "build_ngh": n * (8 + 4 + 1) + cells * (4 + 8 + 16 + 100),   # xy, point_cell, is_core; cells, ngh
        "core_mark": n * (8 + 1) + cells * (100 + 4 + 1 + 4),        # xy, is_core; ngh, start, status, uf
        "union_find": n * (8 + 1) + cells * (100 + 16 + 1 + 4),      # xy, is_core; ngh, bbox, status, uf
        "cluster_id": cells * (4 + 1 + 4 + 4),                       # uf r/w, status, rank
        "core_labels": 0,
        "border_assign": n * (8 + 1 + 4 + 4) + cells * (100 + 4 + 4),  # xy, is_core, perm, labels
        "unpermute": 0,
    }


def ncu_traffic(kernels):
    """DRAM bytes (read + write) of one launch of each of `kernels`, summed,
    from the committed ncu summary of this workload (its table gives MB read
    and written per kernel); None unless every kernel has a row."""
    found = {}
    try:
        with open(PROFILE_MD) as f:
            for line in f:
                cols = [c.strip() for c in line.strip().strip("|").split("|")]
                if len(cols) > 3 and cols[0] in kernels and cols[0] not in found:
                    found[cols[0]] = (float(cols[2]) + float(cols[3])) * 1e6
    except (OSError, ValueError):
        return None
    if len(found) != len(kernels):
        return None
    return int(round(sum(found.values())))


# ------------------------------------------------------------ baseline legs
def cpu_baseline(X: np.ndarray, eps: float, ms: int, budget_s: float = 15.0):
    """The reference's CPU path (oracle/_ref/cpu) on all host cores, else the
    single-threaded C oracle port; bounded to ~budget_s of CPU work."""
    if ORACLE_DIR not in sys.path:
        sys.path.insert(0, ORACLE_DIR)
    import refmod
    ref = refmod.load("cpu")
    cores = os.cpu_count() or 1
    if ref is not None:
        torch.set_num_threads(cores)
        Xt = torch.from_numpy(X)
        ref.dbscan2d(Xt, eps, ms)  # warm-up
        times = []
        t_end = time.perf_counter() + budget_s
        while len(times) < 3 or (time.perf_counter() < t_end and len(times) < 20):
            t0 = time.perf_counter()
            ref.dbscan2d(Xt, eps, ms)
            times.append(time.perf_counter() - t0)
        kind, used = "reference", torch.get_num_threads()
    else:
        import oracle
        times = []
        t_end = time.perf_counter() + budget_s
        while len(times) < 1 or (time.perf_counter() < t_end and len(times) < 5):
            t0 = time.perf_counter()
            oracle.dbscan2d(X, eps, ms)
            times.append(time.perf_counter() - t0)
        kind, used = "port", 1
    med = statistics.median(times)
    return {"value": round(X.shape[0] / med / 1e6, 3), "unit": UNIT, "cores": used, "kind": kind,
            "sample": f"{len(times)} calls on the full {X.shape[0]:,}-point workload, median "
                      f"{med * 1e3:.1f} ms/call ({cores} host cores visible; fresh process, no GPU work)"}


def reference_cuda_leg(X_np: np.ndarray, steps: int, warmup: int, labels_out: str):
    """The reference's CUDA build (oracle/_ref/cuda) timed like this build:
    W warm-up calls, then `steps` calls each bracketed by CUDA events on the
    current stream, a 512 MB buffer written between calls outside the events;
    plus the median of three dbscan2d_profile stage splits. Labels of the last
    call go to `labels_out` (.npy) for the parent to compare."""
    if ORACLE_DIR not in sys.path:
        sys.path.insert(0, ORACLE_DIR)
    import refmod
    ref = refmod.load("cuda")
    if ref is None:
        return {"unavailable": "reference CUDA build not present in oracle/_ref/cuda"}
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    X = torch.from_numpy(X_np).to(dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    lab = None
    for _ in range(max(3, warmup)):
        lab = ref.dbscan2d(X, EPS, MIN_SAMPLES)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        lab = ref.dbscan2d(X, EPS, MIN_SAMPLES)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in ev]
    profs = []
    for k in range(3):
        flush.fill_(float(k))
        profs.append(ref.dbscan2d_profile(X, EPS, MIN_SAMPLES)[1])
    stage = {s: round(statistics.median(p[s] for p in profs), 4) for s in profs[0]}
    np.save(labels_out, lab.cpu().numpy())
    mean = sum(ms) / len(ms)
    return {"ms_per_step": round(mean, 4), "median_ms": round(statistics.median(ms), 4),
            "value": round(X_np.shape[0] / (mean * 1e-3) / 1e6, 2), "unit": UNIT, "steps": steps,
            "stage_ms": stage,
            "build": "reference csrc/ (extension.cpp, cpu/dbscan_cpu.cpp, cuda/dbscan_cuda.cu) built "
                     "by oracle/build_ref.py: nvcc -O3 --use_fast_math, TORCH_CUDA_ARCH_LIST=10.0"}


def _child_leg(leg: str, points: str, extra=()) -> dict:
    """Runs one baseline leg of this script in a fresh child process and
    returns its JSON line (or an object saying why there is none)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--leg", leg, "--points-file", points, *extra]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    except subprocess.TimeoutExpired:
        return {"unavailable": f"{leg} leg timed out"}
    for line in reversed(r.stdout.splitlines()):
        if line.startswith("{"):
            return json.loads(line)
    return {"unavailable": f"{leg} leg exited {r.returncode}: {r.stderr.strip()[-300:]}"}


def run_leg(args):
    X = np.load(args.points_file)
    if args.leg == "cpu":
        return cpu_baseline(X, EPS, MIN_SAMPLES)
    return reference_cuda_leg(X, args.steps, args.warmup, args.labels_out)


# ------------------------------------------------------------------- setup
def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------- reference arm
def run_reference(args, world, rank):
    """The reference's own CPU implementation on this workload: imports the
    generators (by file) and the reference's module, nothing of this build."""
    if rank != 0:
        return None
    X = _synthetic().constant_density(N_POINTS, seed=0)
    base = cpu_baseline(X, EPS, MIN_SAMPLES, budget_s=max(10.0, 2.0 * args.steps))
    return {"metric": METRIC, "value": base["value"], "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(N_POINTS / (base["value"] * 1e6) * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": DATA, "config": base_config(world), "device": "host CPU",
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


# ----------------------------------------------------------------- our arm
def run_ours(args, world, rank, local):
    syn = _synthetic()
    X_np = getattr(syn, GENERATOR)(N_POINTS, seed=rank)

    # Baseline legs first, each in a fresh child process, before this process
    # touches the GPU or loads this build.
    legs = {}
    tmpdir = None
    if rank == 0 and world == 1 and not (args.no_cpu_baseline and args.no_reference_cuda):
        tmpdir = tempfile.mkdtemp(prefix="dbs_bench_")
        pts = os.path.join(tmpdir, "points.npy")
        np.save(pts, X_np)
        if not args.no_cpu_baseline:
            legs["cpu"] = _child_leg("cpu", pts)
        if not args.no_reference_cuda:
            legs["ref_cuda"] = _child_leg("ref_cuda", pts, ["--steps", str(args.steps), "--warmup",
                                                            str(args.warmup), "--labels-out",
                                                            os.path.join(tmpdir, "ref_labels.npy")])

    torch.cuda.set_device(local)
    pkg = _package()
    _C, dbscan2d = pkg._C, pkg.dbscan2d
    dev = torch.device("cuda", local)
    X = torch.from_numpy(X_np).to(dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    # Shape and work counts of the pipeline on this input.
    _, info = _C.dbscan2d_info(X, EPS, MIN_SAMPLES)
    # Warm-up as the timed loop runs: each result held until the next call
    # returns, so both label buffers the loop alternates between have their
    # launch graph recorded before timing starts.
    labels = None
    for _ in range(max(3, args.warmup)):
        labels = dbscan2d(X, EPS, MIN_SAMPLES)
    _C.check_status()

    barrier(world)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            labels = dbscan2d(X, EPS, MIN_SAMPLES)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    barrier(world)
    _C.check_status()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    step_stats = {"min": round(min(step_ms), 4), "median": round(statistics.median(step_ms), 4),
                  "max": round(max(step_ms), 4)}
    ms_mean = sum(step_ms) / len(step_ms)
    ms_max = max_over_ranks(ms_mean, world)
    value = world * N_POINTS / (ms_max * 1e-3) / 1e6
    ours_labels = labels.cpu().numpy()

    # Per-stage split (profile entry point: CUDA events between stages).
    prof_runs = []
    for k in range(3):
        flush.fill_(float(k))
        _, prof = _C.dbscan2d_profile(X, EPS, MIN_SAMPLES)
        prof_runs.append(prof)
    prof = {s: statistics.median(r[s] for r in prof_runs) for s in prof_runs[0]}
    cells, passes, kb = info["num_cells"], info["passes"], info["key_bytes"]
    sb = stage_bytes(N_POINTS, cells, passes, kb)
    dom = max(STAGE_LAUNCHES, key=lambda s: prof[s])
    form = info["sort_form"]
    stage_kernels = dict(STAGE_KERNEL, sort_gather=SORT_KERNELS[form])
    kernels = stage_kernels.get(dom, (dom,))
    kernel = "+".join(kernels)
    peak, peak_kind = _peaks()
    # The stage's kernels (one launch each) do its work; the stage time also
    # holds the launches that return at once (a few microseconds).
    achieved = sb[dom] / (prof[dom] * 1e-3) / 1e9
    b_alg_total = sum(sb.values())
    roof = {"bound": "hbm", "kernel": kernel, "stage": dom, "launches": STAGE_LAUNCHES[dom],
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": peak_kind,
            "alg_bytes_per_launch": sb[dom],
            "traffic": ncu_traffic(kernels) if dom in stage_kernels else None,
            "pipeline_alg_bytes": b_alg_total,
            "pipeline_frac": round(b_alg_total / (ms_mean * 1e-3) / 1e9 / peak, 4),
            "stage_ms": {s: round(v, 4) for s, v in prof.items()},
            "stage_frac": {s: round(sb[s] / (prof[s] * 1e-3) / 1e9 / peak, 4)
                           for s in STAGE_LAUNCHES if prof[s] > 0}}

    # End to end through the public API with host buffers.
    X_host = torch.from_numpy(X_np).pin_memory()
    # Warm-up keeps each result alive until the next call returns, as the
    # timed loop does, so the caching host allocator holds both pinned label
    # blocks before timing starts.
    lab_host = None
    for _ in range(3):
        lab_host = dbscan2d(X_host, EPS, MIN_SAMPLES)
    e2e_ms = []
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lab_host = dbscan2d(X_host, EPS, MIN_SAMPLES)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_mean = max_over_ranks(sum(e2e_ms) / len(e2e_ms), world)
    assert lab_host.device.type == "cpu"

    out = {"metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max, 4),
           "step_ms": step_stats,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": DATA, "config": base_config(world),
           "pipeline": {"num_cells": cells, "key_bits": info["key_bits"], "radix_passes": passes,
                        "sort": SORT_FORM_NAME[form],
                        "queries": info["queries"], "border_points": info["border"],
                        "union_pairs": [info["pairs_ring0"], info["pairs_ring1"]],
                        "union_warp_pairs": [info["warp_pairs_ring0"], info["warp_pairs_ring1"]]},
           "clocks": clocks.summary(),
           "e2e": {"value": round(world * N_POINTS / (e2e_mean * 1e-3) / 1e6, 2), "unit": UNIT,
                   "h2d_bytes_per_step": N_POINTS * 8, "d2h_bytes_per_step": N_POINTS * 4},
           "gpu_launches": KERNELS_PER_CALL * args.steps,
           "roofline": roof}
    if "cpu" in legs:
        out["cpu_baseline"] = legs["cpu"]
    if "ref_cuda" in legs:
        rc = legs["ref_cuda"]
        if "ms_per_step" in rc:
            ref_lab = np.load(os.path.join(tmpdir, "ref_labels.npy"))
            rc["labels_equal"] = bool(np.array_equal(ref_lab, ours_labels))
            rc["speedup"] = round(rc["ms_per_step"] / ms_mean, 2)  # mean over mean, as `value`
            rc["speedup_median"] = round(rc["median_ms"] / statistics.median(step_ms), 2)
        out["reference_cuda"] = rc
    if tmpdir is not None:
        import shutil
        shutil.rmtree(tmpdir, ignore_errors=True)
    del labels, X, flush, X_host
    torch.cuda.empty_cache()
    if world == 1:
        if not args.no_configs:
            out["configs"] = run_configs(dev)
        if args.batched_clouds > 0:
            out["batched"] = run_batched(dev, args.batched_clouds)
        if args.serve_seconds > 0:
            out["serving"] = run_serving(dev, args.serve_seconds, args.serve_sweep_seconds)
    elif args.batched_clouds > 0:
        out["batched"] = run_batched_sharded(dev, args.batched_clouds, world, rank)
    return out


def _ev_ms(fn):
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    out = fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b), out


def run_batched_sharded(dev, n_clouds: int, world: int, rank: int) -> dict:
    """The batched workload split across ranks by shard_clouds (independent
    clouds, no collective on the data path): each rank clusters its shard in
    one batched run; the time is the max over ranks."""
    pkg = _package()
    sizes, eps, ms = _synthetic().batch_layout(n_clouds, seed=0)
    mine = pkg.shard_clouds(sizes, world)[rank]
    X, off = _synthetic().blobs_with_noise_device(sizes[mine], seed=rank, device=dev)
    pkg.dbscan2d_batched(X, off, eps[mine], ms[mine])  # warm-up
    tb = [_ev_ms(lambda: pkg.dbscan2d_batched(X, off, eps[mine], ms[mine]))[0] for _ in range(3)]
    pkg.check_status()
    t = max_over_ranks(statistics.median(tb), world)
    del X
    torch.cuda.empty_cache()
    return {"workload": f"{n_clouds} clouds sharded over {world} ranks (longest-first greedy by points)",
            "clouds": n_clouds, "points": int(sizes.sum()), "batched_ms": round(t, 3),
            "batched_clouds_per_s": round(n_clouds / (t * 1e-3), 1),
            "batched_mpoints_per_s": round(int(sizes.sum()) / (t * 1e-3) / 1e6, 1)}


def run_batched(dev, n_clouds: int) -> dict:
    """The batched workload: n_clouds independent clouds (sizes log-uniform in [256, 262144],
    eps_i in [0.2, 1.0], min_samples_i in {4..32}) clustered by one batched
    pipeline run, against a loop of plain calls over the same device-resident
    clouds. Both timed with CUDA events; labels compared cloud by cloud.
    Then the same batch through a BatchedPlan (CUDA graph replay) with the
    built-in launch shape and with the shape BatchedPlan.tune() picks."""
    pkg = _package()
    dbscan2d, dbscan2d_batched = pkg.dbscan2d, pkg.dbscan2d_batched
    sizes, eps, ms = _synthetic().batch_layout(n_clouds, seed=0)
    X, off = _synthetic().blobs_with_noise_device(sizes, seed=0, device=dev)
    offl = off.tolist()
    dbscan2d_batched(X, off, eps, ms)  # warm-up
    tb = []
    for _ in range(3):
        t, lab_b = _ev_ms(lambda: dbscan2d_batched(X, off, eps, ms))
        tb.append(t)

    def loop():
        return [dbscan2d(X[offl[k]:offl[k + 1]], float(eps[k]), int(ms[k])) for k in range(n_clouds)]

    loop()  # warm-up: the caching allocator holds every workspace size afterwards
    tp, labs = _ev_ms(loop)
    equal = all(torch.equal(labs[k], lab_b[offl[k]:offl[k + 1]]) for k in range(n_clouds))
    pkg.check_status()
    del labs
    torch.cuda.empty_cache()
    plan = pkg.BatchedPlan(offl)
    plan.run(X, eps, ms)  # captures the graph (built-in shape)
    t_plan = statistics.median([_ev_ms(plan.run)[0] for _ in range(3)])
    gaps = graph_gaps(plan, t_plan)
    t0 = time.perf_counter()
    tuned = plan.tune()
    tune_s = time.perf_counter() - t0
    plan.run()  # captures the graph with the tuned shape
    t_tuned = statistics.median([_ev_ms(plan.run)[0] for _ in range(3)])
    equal_tuned = torch.equal(plan.labels, lab_b)
    if plan.status() != 0:
        raise RuntimeError("batched plan: device status non-zero")
    t_b = statistics.median(tb)
    n_pts = int(offl[-1])
    del X, lab_b, plan
    torch.cuda.empty_cache()
    return {"workload": f"{n_clouds} clouds, N_i log-uniform [256, 262144], eps_i U[0.2, 1.0], "
                        f"min_samples_i U{{4..32}} (device generator, seed 0)",
            "clouds": n_clouds, "points": n_pts,
            "batched_ms": round(t_b, 3), "batched_clouds_per_s": round(n_clouds / (t_b * 1e-3), 1),
            "batched_mpoints_per_s": round(n_pts / (t_b * 1e-3) / 1e6, 1),
            "plain_loop_ms": round(tp, 3), "plain_loop_clouds_per_s": round(n_clouds / (tp * 1e-3), 1),
            "speedup": round(tp / t_b, 2), "labels_equal": bool(equal),
            "plan": {"graph_ms": round(t_plan, 3), "tuned_graph_ms": round(t_tuned, 3),
                     "tuned_shape": dict(zip(("count", "cell_prep", "core", "pairs", "pair_scan", "labels"),
                                             tuned["shape"])),
                     "builtin_shape": list(tuned["default_shape"]),
                     "tune_s": round(tune_s, 2), "shapes_timed": tuned["trials"],
                     "labels_equal": bool(equal_tuned), "launch_gaps": gaps}}


def graph_gaps(plan, graph_ms: float) -> dict:
    """Launch gaps inside one replay of the plan's graph: the kernels' own
    durations (a CUPTI trace of one replay through torch.profiler) against
    the replay's CUDA-event time measured without the profiler. The
    difference bounds what one persistent launch of the whole pipeline could
    save."""
    torch.cuda.synchronize()
    with torch.profiler.profile(activities=[torch.profiler.ProfilerActivity.CUDA]) as prof:
        plan.run()
        torch.cuda.synchronize()
    kern = [e for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA
            and ("k_" in e.name or "dbs::" in e.name)]
    ksum = sum(e.device_time_total for e in kern) / 1e3  # us -> ms
    return {"kernels": len(kern), "kernel_sum_ms": round(ksum, 3), "graph_ms": round(graph_ms, 3),
            "gap_ms": round(graph_ms - ksum, 3),
            "gap_per_launch_us": round((graph_ms - ksum) * 1e3 / max(1, len(kern)), 2)}


def run_configs(dev) -> dict:
    """The other plain-call workloads, device-resident, CUDA events around each
    call (median of 7 after 3 warm-ups): 100k blobs with noise, constant density
    at 1M and 5M points, the adversarial 4M cloud (min_samples
    4 and 32)."""
    pkg = _package()
    syn = _synthetic()
    dbscan2d = pkg.dbscan2d
    cases = [("blobs_100k", lambda: syn.blobs_with_noise(100_000, seed=0), 0.5, 10),
             ("constant_density_1M", lambda: syn.constant_density(1_000_000, seed=0), 0.5, 10),
             ("constant_density_5M", lambda: syn.constant_density(5_000_000, seed=0), 0.5, 10),
             ("adversarial_4M_ms4", lambda: syn.adversarial(4_000_000, seed=0), 0.5, 4),
             ("adversarial_4M_ms32", None, 0.5, 32)]
    out = {}
    X = None
    for name, gen, eps, ms in cases:
        if gen is not None:
            X = torch.from_numpy(gen()).to(dev)
        for _ in range(3):
            dbscan2d(X, eps, ms)
        ts = [_ev_ms(lambda: dbscan2d(X, eps, ms))[0] for _ in range(7)]
        t = statistics.median(ts)
        out[name] = {"n_points": int(X.shape[0]), "eps": eps, "min_samples": ms, "ms": round(t, 4),
                     "mpoints_per_s": round(X.shape[0] / (t * 1e-3) / 1e6, 1)}
    pkg.check_status()
    del X
    torch.cuda.empty_cache()
    return out


# ----------------------------------------------------------------- serving
SERVE_RATE_HZ = 2000.0
SERVE_BUDGET = 64 << 30
P99_BOUND_MS = 50.0
SERVE_WARMUP_S = 3.0


class RequestPool:
    """Host-side request clouds of the blobs-with-noise distribution: `bases` clouds
    of `base_n` points (20 blobs + 5% noise, shuffled; device generator, one
    seed per cloud) copied once to pinned host memory. Request i is the
    window of its size at a seeded random offset of base cloud i mod bases:
    a random subsample of a shuffled blobs-with-noise cloud, so such a cloud of
    that size, and no two requests share their point set."""

    def __init__(self, dev, bases: int = 64, base_n: int = 2_000_000, seed: int = 1):
        X, _ = _synthetic().blobs_with_noise_device([base_n] * bases, seed=seed, device=dev)
        self.host = X.cpu().pin_memory()
        del X
        torch.cuda.empty_cache()
        self.bases, self.base_n = bases, base_n

    def windows(self, sizes, seed):
        rng = np.random.default_rng(seed)
        off = rng.integers(0, self.base_n - np.asarray(sizes) + 1)
        return [self.host[(i % self.bases) * self.base_n + int(o):
                          (i % self.bases) * self.base_n + int(o) + int(n)]
                for i, (o, n) in enumerate(zip(off, sizes))]


def _serve(srv, xs, arrivals, eps, ms, keep_every=0):
    """Offers the requests to the server at their arrival times (host
    clock); returns (latencies ms, clouds/s from the first arrival to the last
    completion, batches, {request index: labels} of every keep_every-th
    request). Finished requests are released as they complete (a caller
    holding every result would pin one label buffer per request)."""
    n = len(xs)
    srv.batches = srv.completed = 0
    lat = np.empty(n)
    kept = {}
    pending = {}
    srv.pop_finished()
    t0 = time.perf_counter()
    t_last = t0
    i = 0
    while i < n or pending:
        now = time.perf_counter() - t0
        while i < n and arrivals[i] <= now:
            r = srv.submit(xs[i], float(eps[i]), int(ms[i]), t_submit=t0 + arrivals[i])
            pending[r.rid] = i
            i += 1
        if srv.step() == 0:
            time.sleep(20e-6)
        else:
            for r in srv.pop_finished():
                k = pending.pop(r.rid)
                lat[k] = r.latency * 1e3
                t_last = max(t_last, r.t_done)
                if keep_every and k % keep_every == 0:
                    kept[k] = r.labels.clone()  # a view would hold its batch's block
    return lat, n / (t_last - t0), srv.batches, kept


def _plain(dbscan2d, xs, arrivals, eps, ms, keep_every=0):
    """Sequential plain calls (CPU tensor in, labels back on the host) in
    arrival order, each started at its arrival time or when the previous one
    finished; returns (latencies ms, clouds/s, kept labels)."""
    n = len(xs)
    lat = np.empty(n)
    kept = {}
    t0 = time.perf_counter()
    for k in range(n):
        while time.perf_counter() - t0 < arrivals[k]:
            pass
        lab = dbscan2d(xs[k], float(eps[k]), int(ms[k]))
        lat[k] = (time.perf_counter() - t0 - arrivals[k]) * 1e3
        if keep_every and k % keep_every == 0:
            kept[k] = lab
    return lat, n / (time.perf_counter() - t0), kept


def _pct(a, q):
    return round(float(np.percentile(a, q)), 3)


def _tail(lat, arrivals):
    """Where the slow requests were: how many took over the p99 bound, and
    the arrival second of the slowest."""
    k = int(np.argmax(lat))
    return {"max_ms": round(float(lat[k]), 3), "max_at_s": round(float(arrivals[k]), 3),
            "over_bound": int((lat > P99_BOUND_MS).sum())}


def run_serving(dev, seconds: float, sweep_seconds: float) -> dict:
    """Serving: Poisson arrivals at 2,000 req/s for `seconds`, sizes
    log-uniform in [1e3, 2e6] (blobs-with-noise clouds), eps U[0.1, 1.0], min_samples
    U{4..32}, through the continuous-batching server (admission under a 64 GiB
    budget, checked against free device memory) and through sequential plain
    calls, each arm after a SERVE_WARMUP_S warm-up stream at the same rate;
    latency = completion minus arrival (host clock). Then a saturation
    sweep per arm: offered rates rising by sqrt(2) from 1,000 req/s, each for
    `sweep_seconds`, until p99 exceeds 50 ms or the arm falls behind (achieved
    below 95% of offered); the arm's capacity is the highest offered rate that
    stayed within both."""
    pkg = _package()
    syn = _synthetic()
    pool = RequestPool(dev)
    free0, total = torch.cuda.mem_get_info(dev)
    srv = pkg.DbscanServer(budget_bytes=SERVE_BUDGET, lane_points=16 << 20, lane_clouds=256, lanes=3)

    def stream(rate, dur, seed):
        arr, sizes, eps, ms, _ = syn.request_stream(rate_hz=rate, duration_s=dur, seed=seed)
        return arr, pool.windows(sizes, seed + 7), eps, ms, sizes

    # Warm-up of both arms: a stream at the serving rate, so the caching
    # device and pinned-host allocators hold blocks of the request sizes
    # before the timed stream (the first seconds otherwise pay their growth).
    arr, xs, eps, ms, _ = stream(SERVE_RATE_HZ, SERVE_WARMUP_S, 99)
    _serve(srv, xs, arr, eps, ms)
    _plain(pkg.dbscan2d, xs, arr, eps, ms)

    arr, xs, eps, ms, sizes = stream(SERVE_RATE_HZ, seconds, 0)
    # The objects alive before the timed streams (the request views among
    # them) move to the collector's permanent generation, so a full
    # collection during a stream does not walk them: a serving process would
    # freeze its start-up state the same way.
    gc.collect()
    gc.freeze()
    lat_s, cps_s, batches, kept_s = _serve(srv, xs, arr, eps, ms, keep_every=97)
    lat_p, cps_p, kept = _plain(pkg.dbscan2d, xs, arr, eps, ms, keep_every=97)
    equal = kept.keys() == kept_s.keys() and all(torch.equal(kept_s[k], lab) for k, lab in kept.items())
    del kept_s, kept

    def sweep(run_arm):
        steps = []
        rate = 1000.0
        while rate <= 64000.0:
            a, x, e, m, _ = stream(rate, sweep_seconds, int(rate))
            lat, cps = run_arm(x, a, e, m)
            ok = _pct(lat, 99) <= P99_BOUND_MS and cps >= 0.95 * len(x) / max(a[-1], 1e-9)
            steps.append({"offered": round(rate), "achieved": round(cps, 1), "p50_ms": _pct(lat, 50),
                          "p99_ms": _pct(lat, 99), "ok": bool(ok)})
            if not ok:
                break
            rate *= 2 ** 0.5
        good = [s for s in steps if s["ok"]]
        return {"capacity_clouds_per_s": good[-1]["achieved"] if good else 0.0,
                "capacity_offered": good[-1]["offered"] if good else 0, "steps": steps}

    gc.unfreeze()
    srv_arena = srv.arena_bytes
    sat_s = sweep(lambda x, a, e, m: _serve(srv, x, a, e, m)[:2])
    sat_p = sweep(lambda x, a, e, m: _plain(pkg.dbscan2d, x, a, e, m)[:2])
    pkg.check_status()
    host_arena_mb = round(srv.host_arena.bytes / 2**20, 1) if srv.host_arena is not None else 0
    host_fallbacks = srv.host_arena.fallbacks if srv.host_arena is not None else None
    del pool, srv
    torch.cuda.empty_cache()
    ratio = (sat_s["capacity_clouds_per_s"] / sat_p["capacity_clouds_per_s"]
             if sat_p["capacity_clouds_per_s"] else None)
    return {"workload": f"Poisson {SERVE_RATE_HZ:g} req/s for {seconds:g} s (after a {SERVE_WARMUP_S:g} s "
                        f"warm-up stream per arm), N log-uniform [1e3, 2e6] "
                        f"(blobs-with-noise clouds: windows at random offsets of 64 shuffled 2M-point clouds), "
                        f"eps U[0.1, 1.0], min_samples U{{4..32}}",
            "requests": len(xs), "mean_points": round(float(np.mean(sizes)), 1),
            "budget_gb": round(SERVE_BUDGET / 2**30, 1), "free_hbm_gb": round(free0 / 2**30, 1),
            "arena_gb": round(srv_arena / 2**30, 2), "host_arena_mb": host_arena_mb,
            "host_arena_fallbacks": host_fallbacks,
            "server": {"p50_ms": _pct(lat_s, 50), "p99_ms": _pct(lat_s, 99),
                       "clouds_per_s": round(cps_s, 1), "batches": batches, **_tail(lat_s, arr)},
            "sequential_plain": {"p50_ms": _pct(lat_p, 50), "p99_ms": _pct(lat_p, 99),
                                 "clouds_per_s": round(cps_p, 1), **_tail(lat_p, arr)},
            "labels_equal_sampled": bool(equal),
            "saturation": {"p99_bound_ms": P99_BOUND_MS, "step_seconds": sweep_seconds,
                           "server": sat_s, "sequential_plain": sat_p,
                           "capacity_ratio": round(ratio, 2) if ratio else None}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip the timing of the reference's CUDA build")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the timings of the other plain-call workloads")
    ap.add_argument("--batched-clouds", type=int, default=4096,
                    help="clouds of the batched comparison (0 skips it)")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="length of the serving stream (0 skips serving)")
    ap.add_argument("--serve-sweep-seconds", type=float, default=3.0,
                    help="length of each offered-rate step of the saturation sweep")
    ap.add_argument("--workload", choices=["constant_density", "sparse_uniform", "blobs_with_noise"],
                    default="constant_density",
                    help="main workload generator (sparse_uniform, or blobs_with_noise at small sizes: "
                         "the radix-sort path, for profiler captures; the benchmark line is "
                         "constant_density)")
    ap.add_argument("--points", type=int, default=N_POINTS,
                    help="points of the main constant-density workload (smaller clouds for "
                         "profiler captures; the benchmark line is the 10M-point cloud)")
    ap.add_argument("--leg", choices=["cpu", "ref_cuda"], help=argparse.SUPPRESS)
    ap.add_argument("--points-file", help=argparse.SUPPRESS)
    ap.add_argument("--labels-out", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.points != N_POINTS or args.workload != "constant_density":
        globals().update(N_POINTS=int(args.points), WORKLOAD=f"{args.workload}_{int(args.points)}",
                         GENERATOR=args.workload)
    if args.leg:
        print(json.dumps(run_leg(args)), flush=True)
        return
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            out = run_reference(args, world, rank)
        else:
            out = run_ours(args, world, rank, local)
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
