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
# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) per
# algorithmic byte of the partition and the split-scan kernel groups, over
# every launch of one profiled 16-tree fit of this workload
PARTITION_DRAM_PER_ALGORITHMIC_BYTE = 0.71
SCAN_DRAM_PER_ALGORITHMIC_BYTE = 1.00


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
    """The slowest rank's time (replicas: every rank fits its own forest)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(rank: int) -> int:
    """Each replica grows its own forest (different trees per rank)."""
    return 1000 + rank


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- reference
def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def sklearn_fit_seconds(x, y, n_trees, cores):
    from sklearn.ensemble import RandomForestClassifier as SkRF
    rf = SkRF(n_estimators=n_trees, max_features=MAX_FEATURES, bootstrap=True, n_jobs=cores, random_state=0)
    t0 = time.perf_counter()
    rf.fit(x, y)
    return time.perf_counter() - t0


def run_reference(args, world, rank):
    """hybridforest's CPU classifier (builder.py:67-69): scikit-learn RF on all
    cores.  Every timed step fits the whole 100-tree forest on the full data;
    the untimed warm-up steps fit one tree per core (thread pool and data
    conversion warmed, a few seconds each), so that the run stays within a
    few minutes."""
    if rank != 0:
        return 0
    from cudatree_b200 import synthetic
    x, y = synthetic.covtype_like()
    cores = len(os.sched_getaffinity(0))
    warm_trees = min(cores, N_TREES)
    for _ in range(args.warmup):
        sklearn_fit_seconds(x, y, warm_trees, cores)
    times = [sklearn_fit_seconds(x, y, N_TREES, cores) for _ in range(args.steps)]
    per_forest = statistics.mean(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": per_forest, "unit": "s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_forest * 1000, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "form": "scikit-learn RandomForestClassifier (hybridforest CPU path)",
                   "warmup_form": f"{warm_trees}-tree fits (one tree per core)"},
        "cpu_baseline": {"value": per_forest, "unit": "s", "cores": cores, "cpu": cpu_model(), "kind": "reference",
                         "sample": f"the whole {N_TREES}-tree forest on the full 581012x54 data every step, "
                                   f"n_jobs={cores}; min {min(times):.2f} s, max {max(times):.2f} s"},
        "e2e": {"value": per_forest, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------ other configs
def _sk_fit_s(x, y, trees, max_features, bootstrap, cores):
    from sklearn.ensemble import RandomForestClassifier as SkRF
    rf = SkRF(n_estimators=trees, max_features=max_features, bootstrap=bootstrap, n_jobs=cores, random_state=0)
    t0 = time.perf_counter()
    rf.fit(x, y)
    return time.perf_counter() - t0, rf


def _fit_pair(x, y, n_trees, m, bootstrap, bfs_threshold, seed, plain_trees, tuned=None):
    """Batched fit seconds (warm, CUDA events), plain fit seconds on plain_trees
    trees scaled to n_trees, and whether plain grew the same trees."""
    import torch

    from cudatree_b200 import RandomForestClassifier, _lib
    f = RandomForestClassifier(n_trees, max_features=m, bootstrap=bootstrap, seed=seed)
    f.fit_init(x, y)
    f._tuned = tuned
    thr = f.bfs_threshold if bfs_threshold is None else bfs_threshold
    f._fit_trees(0, n_trees, "batched", thr)  # warm-up
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    trees = f._fit_trees(0, n_trees, "batched", thr)
    e1.record(st)
    torch.cuda.synchronize()
    batched_s = e0.elapsed_time(e1) / 1000.0
    f.profile = True
    f._fit_trees(0, n_trees, "batched", thr)
    stats = f.last_fit_stats
    f.profile = False
    t0 = time.perf_counter()
    ptrees = f._fit_trees(0, plain_trees, "plain", thr)
    torch.cuda.synchronize()
    plain_s = (time.perf_counter() - t0) * n_trees / plain_trees
    same = all(np.array_equal(a.left_children, b.left_children) and
               np.array_equal(a.feature_threshold_array, b.feature_threshold_array) and
               np.array_equal(a.values_array, b.values_array) for a, b in zip(ptrees, trees))
    f.fit_release()
    gi = {g: i for i, g in enumerate(_lib.KERNEL_GROUPS)}
    gbs = {g: round(stats["bytes"][gi[g]] / (stats["ms"][gi[g]] * 1e6), 1) if stats["ms"][gi[g]] > 0 else None
           for g in ("scan", "partition")}
    return batched_s, plain_s, same, gbs, sum(t.n_nodes for t in trees)


def run_configs(args):
    """The reference's other configurations: digits-shaped (1,797 x 64, 50
    trees, no bootstrap, bfs_threshold 4196), wide (10,000 x 3,000, 100
    classes, 200 trees, max_features 55, uint16 indices) and the queue of 256
    uneven jobs (10 trees each), each beside scikit-learn on the same host."""
    from cudatree_b200 import RandomForestClassifier, synthetic
    from cudatree_b200.serving import fit_forests
    cores = len(os.sched_getaffinity(0))
    out = {}
    x, y = synthetic.digits_like()
    b, p, same, gbs, nodes = _fit_pair(x, y, 50, 8, False, 4196, 11, 50)
    sk, _ = _sk_fit_s(x, y, 50, 8, False, cores)
    out["digits_1797x64_50trees"] = {"batched_fit_s": b, "plain_fit_s": p, "plain_trees_identical": same,
                                     "nodes": nodes, "sklearn_fit_s": sk, "sklearn_cores": cores}
    x, y = synthetic.wide()
    tuner = RandomForestClassifier(200, max_features=55, seed=12)
    t0 = time.perf_counter()
    tuned = tuner.autotune(x, y, sample_trees=32)
    tune_s = time.perf_counter() - t0
    b, p, same, gbs, nodes = _fit_pair(x, y, 200, 55, True, None, 12, 200, tuned)
    sk, _ = _sk_fit_s(x, y, 200, 55, True, cores)
    out["wide_10000x3000_c100_200trees"] = {
        "batched_fit_s": b, "plain_fit_s": p, "plain_trees_identical": same, "nodes": nodes,
        "kernel_GB_per_s": gbs, "autotuned": {k: tuned[k] for k in tuned if k != "best_ms"}, "autotune_s": tune_s,
        "sklearn_fit_s": sk, "sklearn_cores": cores}
    n_jobs = args.queue_jobs
    jobs = [synthetic.blob_job(j) for j in range(n_jobs)]
    fit_forests(jobs, n_estimators=10, seeds=range(n_jobs))  # warm-up: library, graphs and device buffers
    t0 = time.perf_counter()
    forests = fit_forests(jobs, n_estimators=10, seeds=range(n_jobs))
    q_s = time.perf_counter() - t0
    checked = list(range(0, n_jobs, max(1, n_jobs // 8)))
    same = True
    for j in checked:
        solo = RandomForestClassifier(10, seed=j).fit(*jobs[j])
        same &= all(np.array_equal(a.left_children, c.left_children) and
                    np.array_equal(a.feature_threshold_array, c.feature_threshold_array)
                    for a, c in zip(forests[j]._trees, solo._trees))
    sample = min(16, n_jobs)
    sk = sum(_sk_fit_s(jobs[j][0], jobs[j][1], 10, int(np.ceil(np.sqrt(jobs[j][0].shape[1]))), True, cores)[0]
             for j in range(sample))
    out[f"queue_{n_jobs}_jobs_10trees"] = {
        "total_s": q_s, "jobs_per_s": n_jobs / q_s,
        "form": "ct_fit_queue: jobs grouped by index/label width, each group one shared level loop",
        "level_launches": forests[0].last_fit_stats["total_launches"] if forests[0].last_fit_stats else None,
        "trees_identical_to_solo_fits": bool(same), "checked_jobs": len(checked),
        "sklearn_sample_s": sk, "sklearn_sample": f"jobs 0-{sample - 1} one after another",
        "sklearn_sequential_s_estimate": sk * n_jobs / sample, "sklearn_cores": cores}
    return out


# ------------------------------------------------------------------ serving
def run_serving(args, x_cov, y_cov, seed):
    """Serving workload: a 500-tree covtype-shaped forest + 8 resident forests
    (50-500 trees, 16-512 features), Poisson arrivals at args.rate req/s,
    rows log-uniform in [1, 65536], 5 % small fit jobs (<= 20,000 rows, 10
    trees); p50/p99 latency and rows/s from the engine, and a spot check that
    served predictions equal the plain predict path."""
    import torch

    from cudatree_b200 import RandomForestClassifier
    from cudatree_b200.serving import ForestServer, pinned

    rng = np.random.default_rng(5)
    forests, pools = [], []
    big = RandomForestClassifier(args.serve_trees, max_features=MAX_FEATURES, seed=seed + 17).fit(x_cov, y_cov)
    forests.append(big)
    pools.append(x_cov[:65536])
    feats = [16, 32, 64, 128, 192, 256, 384, 512]
    for j, f in enumerate(feats):
        n, c = 20000, int(rng.integers(2, 51))
        yj = rng.integers(0, c, size=n)
        means = rng.normal(0.0, 1.0, size=(c, f)).astype(np.float32)
        xj = (rng.standard_normal((n, f)).astype(np.float32) + means[yj])
        trees = int(rng.integers(50, 501))
        forests.append(RandomForestClassifier(trees, seed=seed + j).fit(xj, yj))
        pool = (rng.standard_normal((65536, f)).astype(np.float32) + means[rng.integers(0, c, 65536)])
        pools.append(pool)
    # plain-path throughput: one 65,536-row batch on the 500-tree forest
    nodes, offs, compact = big._device_forest()
    from cudatree_b200 import _lib
    fn = "ct_predict_compact" if compact else "ct_predict"
    xd = torch.from_numpy(pools[0]).cuda()
    out = torch.empty(xd.shape[0], dtype=torch.int32, device="cuda")
    votes = torch.empty((xd.shape[0], big.n_labels), dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream()
    n_nodes = nodes.numel() // (8 if compact else 16)
    for _ in range(2):
        _lib.call(fn, nodes.data_ptr(), n_nodes, offs.data_ptr(), len(big._trees), xd.data_ptr(), xd.shape[0],
                  big.n_features, big.n_labels, votes.data_ptr(), out.data_ptr(), st.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    reps = 5
    for _ in range(reps):
        _lib.call(fn, nodes.data_ptr(), n_nodes, offs.data_ptr(), len(big._trees), xd.data_ptr(), xd.shape[0],
                  big.n_features, big.n_labels, votes.data_ptr(), out.data_ptr(), st.cuda_stream)
    e1.record(st)
    torch.cuda.synchronize()
    batch_rows_per_s = reps * xd.shape[0] / (e0.elapsed_time(e1) / 1000.0)

    srv = ForestServer(max_features=512, fit_workers=2, max_fit_rows=20000, max_fit_trees=10)
    ids = [srv.add_forest(f) for f in forests]
    pinned_pools = [pinned(p) for p in pools]
    fit_x, fit_y = pinned(pools[3][:20000]), pinned(rng.integers(0, 10, 20000).astype(np.uint32))
    n_req = int(args.rate * args.serve_seconds)
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, size=n_req))
    reqs, meta = [], []
    rows_total = 0
    plans = []
    for i in range(n_req):
        if rng.random() < args.fit_frac:
            n = int(np.exp(rng.uniform(np.log(500), np.log(20000))))
            plans.append(("fit", n))
        else:
            k = int(rng.integers(0, len(forests)))
            n = int(np.exp(rng.uniform(0.0, np.log(65536))))
            plans.append(("predict", k, n, int(rng.integers(0, 65536 - n + 1))))
            rows_total += n
    outbuf = torch.zeros(rows_total, dtype=torch.int32).pin_memory()
    pos = 0
    for i, plan in enumerate(plans):
        if plan[0] == "fit":
            n = plan[1]
            r = srv.fit_request(fit_x[:n], fit_y[:n], n_classes=10, n_trees=10, seed=i)
            meta.append(None)
        else:
            _, k, n, lo = plan
            xs = pinned_pools[k][lo:lo + n]
            o = outbuf[pos:pos + n]
            r = srv.predict_request(ids[k], xs, o)
            meta.append((k, lo, n, pos))
            pos += n
        r.arrival_s = float(arrivals[i])
        reqs.append(r)
    stats = srv.replay(reqs, timeout_s=300.0)
    # spot check: served predictions == plain predict path
    same = True
    checked = 0
    for i in rng.permutation(len(reqs))[:40]:
        if meta[i] is None or reqs[i].status != 0:
            continue
        k, lo, n, p0 = meta[i]
        got = forests[k].compt_table[outbuf[p0:p0 + n].numpy().astype(np.int64)]
        same &= bool(np.array_equal(got, forests[k].predict(pools[k][lo:lo + n])))
        checked += 1
    srv.close()
    return {
        "workload": f"{args.serve_trees}-tree covtype-shaped forest + 8 forests (50-500 trees, 16-512 features); "
                    f"Poisson {args.rate:g} req/s for {args.serve_seconds:g} s, rows log-uniform [1, 65536], "
                    f"{100 * args.fit_frac:g}% fit jobs (<= 20000 rows, 10 trees)",
        "requests": int(stats["requests"]), "fit_jobs": int(stats["fit_jobs"]), "rejected": int(stats["rejected"]),
        "rows_per_s": stats["rows_per_s"], "p50_ms": stats["p50_ms"], "p99_ms": stats["p99_ms"],
        "p50_ms_le4096_rows": stats["p50_small_ms"], "p99_ms_le4096_rows": stats["p99_small_ms"],
        "p50_fit_ms": stats["p50_fit_ms"], "p99_fit_ms": stats["p99_fit_ms"], "batches": int(stats["batches"]),
        "zero_copy_requests": int(stats["zero_copy_requests"]),
        "hbm_used_gb": stats["hbm_used_bytes"] / 1e9,
        "identical_to_plain_predict": bool(same), "checked_requests": checked,
        "plain_predict_rows_per_s_500_trees": batch_rows_per_s,
    }


def run_predict_only(args):
    """Plain predict throughput on a forest fit to the covtype-shaped data:
    65,536-row batches through ct_predict (packed nodes) and
    ct_predict_compact (8-byte nodes), with and without the vote table (the
    table lets the launch walk L2-sized tree groups)."""
    import torch

    from cudatree_b200 import RandomForestClassifier, _lib, synthetic
    x, y = synthetic.covtype_like()
    forest = RandomForestClassifier(args.serve_trees, max_features=MAX_FEATURES, seed=77).fit(x, y)
    xd = torch.from_numpy(x[:65536]).cuda()
    out = torch.empty(xd.shape[0], dtype=torch.int32, device="cuda")
    votes = torch.empty((xd.shape[0], forest.n_labels), dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream()
    res = {}
    for name, vt, compact in (("packed_no_vote_table", None, False), ("packed_tree_groups", votes, False),
                              ("compact_no_vote_table", None, True), ("compact_tree_groups", votes, True)):
        nodes, offs, _ = forest._device_forest(compact)

        n_nodes = nodes.numel() // (8 if compact else 16)

        def call():
            _lib.call("ct_predict_compact" if compact else "ct_predict", nodes.data_ptr(), n_nodes,
                      offs.data_ptr(), len(forest._trees), xd.data_ptr(), xd.shape[0], forest.n_features,
                      forest.n_labels, None if vt is None else vt.data_ptr(), out.data_ptr(), st.cuda_stream)
        for _ in range(args.warmup):
            call()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            call()
        e1.record(st)
        torch.cuda.synchronize()
        res[name] = args.steps * xd.shape[0] / (e0.elapsed_time(e1) / 1000.0)
    print(json.dumps({"predict_rows_per_s": res, "trees": args.serve_trees,
                      "nodes": int(sum(t.n_nodes for t in forest._trees))}), flush=True)
    return 0


# --------------------------------------------------------------------- ours
def run_ours(args, world, rank, local):
    import torch
    sys.path.insert(0, str(ROOT))
    from cudatree_b200 import RandomForestClassifier, _lib, synthetic

    x, y = synthetic.covtype_like()
    seed = replica_seed(rank)
    n_trees = args.trees
    tune = not args.no_autotune
    forest = RandomForestClassifier(n_trees, max_features=MAX_FEATURES, bootstrap=True, seed=seed, autotune=tune)
    tune_s = None
    if tune:  # the library's autotuner on the whole forest, before anything is timed
        t0 = time.perf_counter()
        forest.autotune(x, y, sample_trees=n_trees)
        tune_s = time.perf_counter() - t0
    forest.fit_init(x, y)
    thr = forest.bfs_threshold
    stream = torch.cuda.current_stream()

    def step(mode="batched", profile=False):
        forest.profile = profile
        return forest._fit_trees(0, n_trees, mode, thr)

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
            trees = step()
            launches += forest.last_fit_stats["total_launches"]
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    step_s = ev0.elapsed_time(ev1) / 1000.0 / args.steps
    job_s = max_over_ranks(step_s, world)
    # per-kernel-group times and algorithmic bytes: one more step, with CUDA
    # events between the groups on the launching stream (outside the timed region)
    step(profile=True)
    torch.cuda.synchronize()
    stats = forest.last_fit_stats
    n_nodes = sum(t.n_nodes for t in trees)

    # plain per-node form on the same forest (one warm-up tree, one timed forest)
    plain_s = None
    if not args.skip_plain:
        forest._fit_trees(0, 1, "plain", thr)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        plain_trees = forest._fit_trees(0, n_trees, "plain", thr)
        torch.cuda.synchronize()
        plain_s = time.perf_counter() - t0
        same = all(np.array_equal(a.left_children, b.left_children) and
                   np.array_equal(a.feature_threshold_array, b.feature_threshold_array) and
                   np.array_equal(a.values_array, b.values_array) for a, b in zip(plain_trees, trees))
    forest.fit_release()

    # end to end through the public API: pinned host arrays in, trees out
    xp = torch.from_numpy(x).pin_memory() if args.e2e_steps > 0 else None
    yp = torch.from_numpy(y)
    e2e_times = []
    f2 = forest
    for i in range(1 + args.e2e_steps if args.e2e_steps > 0 else 0):
        f2 = RandomForestClassifier(n_trees, max_features=MAX_FEATURES, bootstrap=True, seed=seed, autotune=tune)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f2.fit(xp, yp)
        torch.cuda.synchronize()
        if i > 0:
            e2e_times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(statistics.mean(e2e_times), world) if e2e_times else None
    d2h = sum(t.n_nodes for t in trees) * 20 + 4 * n_trees

    serving = None if args.skip_serving else run_serving(args, x, y, seed)
    configs = None if args.skip_configs or rank != 0 else run_configs(args)
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
    pi = groups.index("partition")
    p_ms = stats["ms"][pi]
    p_gbs = stats["bytes"][pi] / (p_ms * 1e6) if p_ms > 0 else None
    # DRAM bytes per partition launch: the algorithmic bytes per launch times
    # the DRAM/algorithmic ratio ncu measured on the 16-tree case of this
    # workload (dram__bytes_read.sum + dram__bytes_write.sum of the partition
    # launches of that capture)
    p_launches = stats["launches"][pi]
    traffic = (PARTITION_DRAM_PER_ALGORITHMIC_BYTE * stats["bytes"][pi] / p_launches) if p_launches else None
    si = groups.index("scan")
    s_ms = stats["ms"][si]
    s_gbs = stats["bytes"][si] / (s_ms * 1e6) if s_ms > 0 else None
    s_launches = stats["launches"][si]
    s_traffic = (SCAN_DRAM_PER_ALGORITHMIC_BYTE * stats["bytes"][si] / s_launches) if s_launches else None
    cpu = None
    if not args.skip_cpu:
        cores = len(os.sched_getaffinity(0))
        t_cpu = sklearn_fit_seconds(x, y, N_TREES, cores)
        cpu = {"value": t_cpu, "unit": "s", "cores": cores, "cpu": cpu_model(), "kind": "reference",
               "sample": f"scikit-learn RandomForestClassifier (hybridforest CPU path): one fit of the whole "
                         f"{N_TREES}-tree forest on the full data, n_jobs={cores}"}
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
        "fit_options": ({k: v for k, v in forest._tuned.items() if k != "sample_ms"} if forest._tuned else "defaults"),
        "autotune_s": tune_s,
        "kernels": kernels,
        "roofline": {"bound": "hbm", "kernel": "k_partition", "achieved": round(p_gbs, 1) if p_gbs else None,
                     "peak": peak, "unit": "GB/s", "frac": round(p_gbs / peak, 4) if p_gbs else None,
                     "peak_kind": peak_kind, "traffic": round(traffic) if traffic else None,
                     "traffic_unit": f"DRAM bytes per launch (ncu ratio {PARTITION_DRAM_PER_ALGORITHMIC_BYTE} x algorithmic, 16-tree capture)",
                     "algorithmic_bytes_per_launch": round(stats["bytes"][pi] / p_launches) if p_launches else None,
                     "algorithmic_bytes_per_element": "n_features x (2 x index_bytes + 1)"},
        "scan_roofline": {"bound": "hbm", "kernel": "k_split_scan (+hist, carry, two-valued, virtual counts)",
                          "achieved": round(s_gbs, 1) if s_gbs else None, "peak": peak, "unit": "GB/s",
                          "frac": round(s_gbs / peak, 4) if s_gbs else None, "peak_kind": peak_kind,
                          "traffic": round(s_traffic) if s_traffic else None,
                          "traffic_unit": f"DRAM bytes per launch (ncu ratio {SCAN_DRAM_PER_ALGORITHMIC_BYTE} x "
                                          f"algorithmic, 16-tree capture)",
                          "algorithmic_bytes_per_launch": round(stats["bytes"][si] / s_launches) if s_launches else None,
                          "algorithmic_bytes_per_element": "per (node, selected feature, position): index_bytes "
                                                           "+ 4 (x gather) + label gather when labels are not packed"},
        "predict": serving,
        "configs": configs,
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
    ap.add_argument("--e2e-steps", type=int, default=2, help="0 skips the end-to-end measurement")
    ap.add_argument("--trees", type=int, default=N_TREES, help="trees per forest (profiling runs use fewer)")
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="fit with the default options (no autotuner)")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-serving", action="store_true")
    ap.add_argument("--predict-only", action="store_true", help="time plain predict only (profiling runs)")
    ap.add_argument("--serve-trees", type=int, default=500)
    ap.add_argument("--serve-seconds", type=float, default=2.0)
    ap.add_argument("--rate", type=float, default=2000.0)
    ap.add_argument("--fit-frac", type=float, default=0.05, help="fraction of serving requests that are fit jobs")
    ap.add_argument("--serving-only", action="store_true", help="run the serving workload alone (profiling runs)")
    ap.add_argument("--skip-configs", action="store_true", help="skip the digits, wide and queue configurations")
    ap.add_argument("--configs-only", action="store_true", help="run only the digits, wide and queue configurations")
    ap.add_argument("--queue-jobs", type=int, default=256)
    args = ap.parse_args()
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        return run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), rank)
    if args.predict_only:
        dist_setup(1)
        return run_predict_only(args)
    if args.configs_only:
        dist_setup(1)
        print(json.dumps({"configs": run_configs(args)}), flush=True)
        return 0
    if args.serving_only:
        dist_setup(1)
        from cudatree_b200 import synthetic
        x, y = synthetic.covtype_like()
        print(json.dumps({"predict": run_serving(args, x, y, 1000)}), flush=True)
        return 0
    world, rank, local = dist_setup(args.gpus)
    try:
        return run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
