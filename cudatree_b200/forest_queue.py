"""Forest queue: many independent small forests through shared launches.

The reference runs a queue of forests as independent fits, one process per
device (``hybridforest/builder.py:79-141``).  Here the jobs are grouped and
each group is one ``ct_fit_queue`` call: every job is prepared on its own
(upload, transpose, presort, label compaction: ``fit_init``), then one node
list holds the nodes of every job's trees and each level step splits them
all, so a group costs one set of level launches instead of one per job.
Each forest is exactly the one ``RandomForestClassifier(n_estimators,
max_features, seed=seeds[i]).fit(x, y)`` grows alone.

Groups: jobs of one index width and label width share a call (the kernels
are compiled per width), and a group's device memory (samples, presort,
index lists, trees) stays within ``group_bytes`` (default 40 % of the free
device memory).  A group's buffers are one allocation; each job is
uploaded, transposed and presorted on the device (the steps of
``fit_init``) before the shared fit, and several groups are fitted side by
side from their own host threads and CUDA streams.
"""
from __future__ import annotations

import ctypes as C
import math
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import _lib
from .random_forest import (PAD_BYTES, RandomForestClassifier, _device, _stream, best_index_bytes, compact_labels,
                            fetch_tree_columns)


def fit_forests(jobs, n_estimators=10, max_features=None, seeds=None, group_bytes=None, fit_options=None,
                streams=4, profile=False):
    """Fit one forest per (x, y) job through shared level steps; returns the
    fitted RandomForestClassifier objects in job order.  fit_options: a dict
    of tuned options (scan_piece, subtree_cutoff, part_shape) for every
    group; the trees do not depend on it.  streams: groups fitted side by
    side, each from its own host thread on its own CUDA stream (the jobs of
    one width are split into at least this many groups of similar size), so
    one group's uploads and level-loop round trips overlap another's kernels.
    profile: CUDA-event time per kernel group in each forest's
    last_fit_stats (its group's)."""
    jobs = [_host_job(x, y, n_estimators, max_features) for x, y in jobs]
    if not jobs:
        return []
    seeds = list(range(len(jobs))) if seeds is None else [int(s) for s in seeds]
    if len(seeds) != len(jobs):
        raise ValueError("one seed per job")
    if group_bytes is None:
        free, _ = torch.cuda.mem_get_info(_device())
        group_bytes = int(0.4 * free)
    streams = max(1, int(streams))
    # groups of one (index width, label width): each within its share of the
    # memory budget (the groups of `streams` threads are in flight at once)
    # and each about 1/streams of its width's bytes.  A group's scratch and
    # class loops are sized by its most classes, so the jobs are ordered by
    # class count and cut into consecutive runs of similar bytes.
    widths = {}
    for i, j in enumerate(jobs):
        widths.setdefault((j.index_bytes, j.label_bytes), []).append(i)
    groups = []
    budget = max(1, group_bytes // streams)
    for members in widths.values():
        total = sum(jobs[i].device_bytes for i in members)
        k = max(min(streams, len(members)), -(-total // budget))
        # cut where the running bytes pass each k-th of the total, so exactly k
        # groups of similar bytes come out (each within the budget when k
        # came from it)
        cur, used, cut = [], 0, 1
        for i in sorted(members, key=lambda i: (jobs[i].c, jobs[i].f)):
            cur.append(i)
            used += jobs[i].device_bytes
            if cut < k and used * k >= cut * total:
                groups.append(sorted(cur))
                cur, cut = [], cut + 1
        if cur:
            groups.append(sorted(cur))
    forests = [None] * len(jobs)
    dev = _device()
    plans = [_GroupPlan([jobs[i] for i in g], fit_options or {}, profile) for g in groups]
    # waves of `streams` groups; a wave's buffers are one allocation (a queue
    # of the same shape later reuses it from the caching allocator)
    for w0 in range(0, len(groups), streams):
        wave = list(range(w0, min(w0 + streams, len(groups))))
        offs, total = {}, 0
        for k in wave:
            offs[k] = total
            total += (plans[k].size + 255) & ~255
        arena = torch.empty(total, dtype=torch.uint8, device=dev)
        torch.cuda.current_stream(dev).synchronize()  # the allocation is ready for the groups' streams

        def run(k):
            g = groups[k]
            st = torch.cuda.Stream(dev)
            with torch.cuda.stream(st):
                res = _fit_group([jobs[i] for i in g], [seeds[i] for i in g], n_estimators, max_features, plans[k],
                                 arena, offs[k], k - w0)
            st.synchronize()
            for i, f in zip(g, res):
                forests[i] = f

        with ThreadPoolExecutor(max_workers=len(wave)) as ex:
            list(ex.map(run, wave))
        del arena
    return forests


class _HostJob:
    """One job's host side: float32 samples, compacted labels and widths."""

    def __init__(self, x, y, n_estimators, max_features):
        x = x.numpy() if isinstance(x, torch.Tensor) else np.asarray(x)
        y = y.numpy() if isinstance(y, torch.Tensor) else np.asarray(y)
        if x.ndim != 2 or y.ndim != 1 or y.shape[0] != x.shape[0] or x.shape[0] == 0:
            raise ValueError("each job is a 2-D samples array and one label per sample")
        self.x = np.ascontiguousarray(x, dtype=np.float32)
        self.table, ids = compact_labels(y)
        self.n, self.f = self.x.shape
        self.c = int(self.table.shape[0])
        if self.c > _lib.MAX_CLASSES or self.f > _lib.MAX_FEATURES - 1:
            raise ValueError("too many classes or features")
        self.index_bytes = best_index_bytes(self.n)
        self.label_bytes = 1 if self.c <= 0xFF else 2
        self.labels = ids.astype(np.uint8 if self.label_bytes == 1 else np.uint16)
        m = int(math.ceil(math.sqrt(self.f))) if max_features is None else int(max_features)
        if not 0 < m <= self.f:
            raise ValueError("max_features must be in [1, n_features]")
        self.m = m
        self.trees = int(n_estimators)
        lists = 2 * self.trees * self.f * self.n * self.index_bytes
        self.device_bytes = (lists + _lib.mark_bytes(self.n, self.trees) + self.f * self.n * (8 + self.index_bytes)
                             + self.n * 2 + self.trees * 2 * self.n * 20 + 8 * 4096)


def _host_job(x, y, n_estimators, max_features):
    return _HostJob(x, y, n_estimators, max_features)


class _Arena:
    """Byte offsets of one group's device buffers (256-aligned, padded for
    the partition's 16-byte bulk copies), carved from one allocation."""

    def __init__(self):
        self.size = 0

    def take(self, nbytes):
        off = (self.size + 255) & ~255
        self.size = off + int(nbytes) + PAD_BYTES
        return off


class _GroupPlan:
    """Offsets of one group's device buffers inside the queue's allocation:
    per job its row-major upload, feature-major samples, labels, presort,
    index lists and marks; NaN flags, the presort workspace, the raw trees
    and the fit's workspace."""

    def __init__(self, jobs, tuned, profile):
        ar = _Arena()
        self.lay = []
        for j in jobs:
            self.lay.append({"x_rm": ar.take(4 * j.n * j.f), "x_fm": ar.take(4 * j.n * j.f),
                             "lab": ar.take(j.labels.nbytes), "pre": ar.take(j.f * j.n * j.index_bytes),
                             "si0": ar.take(j.trees * j.f * j.n * j.index_bytes),
                             "si1": ar.take(j.trees * j.f * j.n * j.index_bytes),
                             "mark": ar.take(_lib.mark_bytes(j.n, j.trees))})
        self.nan = ar.take(4 * len(jobs))
        self.pws = ar.take(max(_presort_ws(j) for j in jobs))
        self.total = sum(j.trees for j in jobs)
        self.cap = 2 * max(j.n for j in jobs)
        self.raw = [ar.take(4 * self.total * self.cap) for _ in range(5)]
        self.n_nodes = ar.take(4 * self.total)
        self.opts = _lib.FitOptions(_lib.CT_FIT_BATCHED, 0, int(tuned.get("subtree_cutoff", 32)),
                                    int(tuned.get("scan_piece", 0)))
        self.opts.part_shape = int(tuned.get("part_shape", 0))
        self.opts.small_rows = int(tuned.get("small_rows", 0))
        if profile:
            self.opts.flags |= _lib.CT_FIT_PROFILE
        self.arr = (_lib.FitJob * len(jobs))()
        for k, j in enumerate(jobs):  # sizes only: the workspace query reads no pointer
            self.arr[k].problem = _lib.Problem(None, None, None, j.n, j.f, j.c, j.index_bytes, j.label_bytes, j.m,
                                               1, 1, 0)
            self.arr[k].lists = _lib.Lists(None, None, None, j.n, j.trees)
            self.arr[k].n_trees = j.trees
        ws = C.c_size_t()
        _lib.call("ct_fit_queue_workspace_size", self.arr, len(jobs), C.byref(self.opts), C.byref(ws))
        self.ws_bytes = ws.value
        self.work = ar.take(ws.value)
        self.size = ar.size


_PINNED = {}  # page-locked upload staging per group slot, kept across calls (grow only)


def _staging(slot: int, nbytes: int) -> torch.Tensor:
    buf = _PINNED.get(slot)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(nbytes, 1), dtype=torch.uint8, pin_memory=True)
        _PINNED[slot] = buf
    return buf


def _fit_group(jobs, seeds, n_estimators, max_features, plan, arena, off, slot):
    """One group's shared fit in arena[off:off + plan.size], on the current
    stream; returns its forests.  slot: the group's page-locked staging."""
    dev = _device()
    mem = arena[off:off + plan.size]
    base = mem.data_ptr()
    lay = plan.lay
    mem[plan.nan:plan.nan + 4 * len(jobs)].zero_()
    mem[plan.n_nodes:plan.n_nodes + 4 * plan.total].zero_()
    # samples and labels to the device: each job is copied into the group's
    # page-locked staging (host) and from there asynchronously on this
    # stream, so the host copy of the next job overlaps this one's transfer
    up = [(j.x.view(np.uint8).reshape(-1), l["x_rm"]) for j, l in zip(jobs, lay)]
    up += [(j.labels.view(np.uint8), l["lab"]) for j, l in zip(jobs, lay)]
    stage = _staging(slot, sum(a.nbytes for a, _ in up))
    host = stage.numpy()
    o = 0
    for a, dst in up:
        host[o:o + a.nbytes] = a
        mem[dst:dst + a.nbytes].copy_(stage[o:o + a.nbytes], non_blocking=True)
        o += a.nbytes
    st = _stream()
    arr = plan.arr
    for k, (j, l) in enumerate(zip(jobs, lay)):
        _lib.call("ct_transpose_rows", base + l["x_rm"], j.n, j.f, base + l["x_fm"], base + plan.nan + 4 * k, st)
        _lib.call("ct_presort", base + l["x_fm"], j.n, j.f, j.index_bytes, base + l["pre"], base + plan.pws,
                  _presort_ws(j), st)
        arr[k].problem = _lib.Problem(base + l["x_fm"], base + l["lab"], base + l["pre"], j.n, j.f, j.c,
                                      j.index_bytes, j.label_bytes, j.m, 1, 1, int(seeds[k]))
        arr[k].lists = _lib.Lists(base + l["si0"], base + l["si1"], base + l["mark"], j.n, j.trees)
        arr[k].n_trees = j.trees
        arr[k].first_tree = 0
    n_nodes = mem[plan.n_nodes:plan.n_nodes + 4 * plan.total].view(torch.int32)
    tb = _lib.TreeBuffers(*[base + r for r in plan.raw], n_nodes.data_ptr(), plan.cap)
    _lib.call("ct_fit_queue", arr, len(jobs), C.byref(plan.opts), C.byref(tb), base + plan.work, plan.ws_bytes, st)
    stats = _lib.fit_stats()
    nan = mem[plan.nan:plan.nan + 4 * len(jobs)].view(torch.int32).cpu().numpy()
    if nan.any():
        raise ValueError(f"samples of job {int(np.flatnonzero(nan)[0])} of the group contain NaN")
    counts, cols = fetch_tree_columns(tb, n_nodes, plan.total, dev)
    out, o, t = [], 0, 0
    for j, seed in zip(jobs, seeds):
        f = RandomForestClassifier(n_estimators, max_features=max_features, seed=seed)
        f.compt_table, f.n_labels, f.n_features, f.n_samples = j.table, j.c, j.f, j.n
        f.dtype_labels = np.dtype(np.uint8 if j.label_bytes == 1 else np.uint16)
        f.index_bytes, f._m, f._seed = j.index_bytes, j.m, int(seed)
        trees = []
        for c in counts[t:t + j.trees].tolist():
            trees.append(f._make_tree(*[col[o:o + c] for col in cols]))
            o += c
        t += j.trees
        f._trees = trees
        f.last_fit_stats = stats
        out.append(f)
    return out


def _presort_ws(j) -> int:
    ws = C.c_size_t()
    _lib.call("ct_presort_workspace_size", j.n, j.f, C.byref(ws))
    return ws.value
