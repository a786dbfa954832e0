"""Benchmark: forest fit on the covtype-shaped workload (581,012 x 54 float32,
7 classes, 100 trees, bootstrap, max_features=7, uint32 indices, fully grown).

One step = one 100-tree forest fit with the batched (level-synchronous) form,
inputs already resident in HBM: bootstrap compaction, tree growth, and the
fitted node arrays read back to the host in canonical order.  The per-node
(plain) form is timed on the same forest, the public API end to end (host
arrays in, trees out), the kernels against the measured HBM roofline, and
the reference's CPU path (hybridforest's CPU classifier: scikit-learn
RandomForestClassifier on all host cores) on a bounded sample.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 each rank fits its own forest (replicas, weak scaling); the time
is the maximum over ranks.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
METRIC = "forest fit s & scan HBM GB/s, batched vs plain; predict rows/s + p50/p99 ms"
WORKLOAD = ("covtype-shaped synthetic 581012x54 f32 (10 Gaussian + 44 one-hot), 7 classes, "
            "100 trees, bootstrap, max_features=7, uint32 indices, fully grown")
N_TREES = 100
MAX_FEATURES = 7


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in Path(self.path).read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def max_over_ranks(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- reference
def sklearn_fit_seconds(x, y, n_trees_sample, cores):
    from sklearn.ensemble import RandomForestClassifier as SkRF
    rf = SkRF(n_estimators=n_trees_sample, max_features=MAX_FEATURES, bootstrap=True, n_jobs=cores,
              random_state=0)
    t0 = time.perf_counter()
    rf.fit(x, y)
    return time.perf_counter() - t0


def run_reference(args, world, rank):
    """hybridforest's CPU classifier (builder.py:67-69): scikit-learn RF on all cores."""
    if rank != 0:
        return 0
    from cudatree_b200 import synthetic
    x, y = synthetic.covtype_like()
    cores = len(os.sched_getaffinity(0))
    sample = min(cores, N_TREES, args.ref_trees)
    for _ in range(args.warmup):
        sklearn_fit_seconds(x, y, sample, cores)
    times = [sklearn_fit_seconds(x, y, sample, cores) for _ in range(args.steps)]
    per_forest = statistics.mean(times) * N_TREES / sample
    line = {
        "impl": "reference", "metric": METRIC, "value": per_forest, "unit": "s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_forest * 1000, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "form": "scikit-learn RandomForestClassifier (hybridforest CPU path)"},
        "cpu_baseline": {"value": per_forest, "unit": "s", "cores": cores, "kind": "reference",
                         "sample": f"{sample} trees per step on the full 581012x54 data, n_jobs={cores}, "
                                   f"scaled x{N_TREES / sample:.2f} to {N_TREES} trees"},
        "e2e": {"value": per_forest, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------- ours
def run_ours(args, world, rank, local):
    import torch
    sys.path.insert(0, str(ROOT))
    from cudatree_b200 import RandomForestClassifier, _lib, synthetic

    x, y = synthetic.covtype_like()
    seed = 1000 + rank
    forest = RandomForestClassifier(N_TREES, max_features=MAX_FEATURES, bootstrap=True, seed=seed)
    forest.fit_init(x, y)
    thr = forest.bfs_threshold
    stream = torch.cuda.current_stream()

    def step(mode="batched", profile=False):
        forest.profile = profile
        return forest._fit_trees(0, N_TREES, mode, thr)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            trees = step(profile=True)
            launches += forest.last_fit_stats["total_launches"]
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    step_s = ev0.elapsed_time(ev1) / 1000.0 / args.steps
    job_s = max_over_ranks(step_s, world)
    stats = forest.last_fit_stats
    n_nodes = sum(t.n_nodes for t in trees)

    # plain per-node form on the same forest (one warm-up tree, one timed forest)
    plain_s = None
    if not args.skip_plain:
        forest._fit_trees(0, 1, "plain", thr)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        plain_trees = forest._fit_trees(0, N_TREES, "plain", thr)
        torch.cuda.synchronize()
        plain_s = time.perf_counter() - t0
        same = all(np.array_equal(a.left_children, b.left_children) and
                   np.array_equal(a.feature_threshold_array, b.feature_threshold_array) and
                   np.array_equal(a.values_array, b.values_array) for a, b in zip(plain_trees, trees))
    forest.fit_release()

    # end to end through the public API: pinned host arrays in, trees out
    xp = torch.from_numpy(x).pin_memory()
    yp = torch.from_numpy(y)
    e2e_times = []
    for i in range(1 + args.e2e_steps):
        f2 = RandomForestClassifier(N_TREES, max_features=MAX_FEATURES, bootstrap=True, seed=seed)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f2.fit(xp, yp)
        torch.cuda.synchronize()
        if i > 0:
            e2e_times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(statistics.mean(e2e_times), world)
    d2h = sum(t.n_nodes for t in f2._trees) * 20 + 4 * N_TREES

    if rank != 0:
        return 0
    peak, peak_kind = peaks()
    groups = _lib.KERNEL_GROUPS
    kernels = {}
    for i, g in enumerate(groups):
        if stats["launches"][i] == 0:
            continue
        ms = stats["ms"][i]
        kernels[g] = {"launches": stats["launches"][i], "ms": round(ms, 3),
                      "GB": round(stats["bytes"][i] / 1e9, 3),
                      "GB_per_s": round(stats["bytes"][i] / (ms * 1e6), 1) if ms > 0 else None}
    part = stats["partition"] if False else None
    pi = groups.index("partition")
    p_ms = stats["ms"][pi]
    p_gbs = stats["bytes"][pi] / (p_ms * 1e6) if p_ms > 0 else None
    traffic = None
    tfile = ROOT / "profiles" / "partition_traffic.json"
    if tfile.exists():
        t = json.loads(tfile.read_text())
        traffic = t.get("dram_bytes_per_algorithmic_byte")
    si = groups.index("scan")
    s_ms = stats["ms"][si]
    cpu = None
    if not args.skip_cpu:
        cores = len(os.sched_getaffinity(0))
        sample = min(cores, N_TREES, args.ref_trees)
        t_cpu = sklearn_fit_seconds(x, y, sample, cores)
        cpu = {"value": t_cpu * N_TREES / sample, "unit": "s", "cores": cores, "kind": "reference",
               "sample": f"scikit-learn RandomForestClassifier (hybridforest CPU path), {sample} trees on the "
                         f"full data, n_jobs={cores}, scaled x{N_TREES / sample:.2f} to {N_TREES} trees"}
    line = {
        "metric": METRIC, "value": job_s, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": job_s * 1000, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 indices, int64 counts, f64 impurity", "data": "synthetic",
        "config": {"workload": WORKLOAD, "form": "batched level-synchronous, all 100 trees in flight",
                   "l2": "inputs larger than L2 (per-tree index lists 2x54x581012x4 B = 251 MB)",
                   "parallelism": f"replicas x{world}"},
        "plain_fit_s": plain_s, "batched_speedup_vs_plain": (plain_s / step_s) if plain_s else None,
        "plain_trees_identical": same if plain_s else None,
        "nodes_per_forest": n_nodes, "level_steps": stats["steps"],
        "kernels": kernels,
        "roofline": {"bound": "hbm", "kernel": "k_partition", "achieved": round(p_gbs, 1) if p_gbs else None,
                     "peak": peak, "unit": "GB/s", "frac": round(p_gbs / peak, 4) if p_gbs else None,
                     "peak_kind": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_element": "n_features x (2 x index_bytes + 1)"},
        "scan_roofline": {"kernel": "k_split_scan (+hist/carry)",
                          "achieved": round(stats["bytes"][si] / (s_ms * 1e6), 1) if s_ms > 0 else None,
                          "peak": peak, "unit": "GB/s"},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(x.nbytes + y.shape[0]),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--ref-trees", type=int, default=100)
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        return run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), rank)
    world, rank, local = dist_setup(args.gpus)
    try:
        return run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
