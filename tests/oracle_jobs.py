"""Oracle trees of the benchmarked configurations, grown in worker processes.

Test infrastructure: the GPU parity tests and the fixture checks submit one
task per tree to a process pool that uses the spawn start method (a pool
forked after the CUDA context exists can hang; the oracle never touches the
GPU).  Each worker regenerates its data set from the seeded synthetic
generators instead of receiving it pickled, and grows the tree with the
oracle's own bootstrap draw and tree key, so a task's tree is exactly tree
``tree`` of ``oracle.fit_forest(x, y, n_estimators, max_features, bootstrap,
min_samples_split, seed)``.
"""
from __future__ import annotations

import functools
import hashlib
import math
import multiprocessing as mp
import os
from concurrent.futures import ProcessPoolExecutor

import numpy as np

from cudatree_b200 import synthetic
from oracle import cudatree_oracle as O


@functools.lru_cache(maxsize=3)
def _data(make: str, arg):
    """(x_fm, compacted labels, n_classes, n_rows, n_features) of a generator."""
    x, y = synthetic.blob_job(arg) if make == "blob_job" else getattr(synthetic, make)()
    x = np.asarray(x, dtype=np.float32)
    classes, yc = O.compact_labels(y)
    return np.ascontiguousarray(x.T), yc, int(classes.shape[0]), x.shape[0], x.shape[1]


def oracle_tree(make: str, arg, tree: int, seed: int, max_features, bootstrap: bool, min_samples_split: int = 1):
    """Tree `tree` of the oracle forest of synthetic.<make>(arg)."""
    x_fm, yc, c, n, f = _data(make, arg)
    m = int(math.ceil(math.sqrt(f))) if max_features is None else int(max_features)
    rows = O.bootstrap_rows(seed, tree, n, bootstrap)
    return O.fit_tree(x_fm, yc, c, rows, m, min_samples_split, O.tree_key(seed, tree))


def pool(workers: int | None = None) -> ProcessPoolExecutor:
    cores = len(os.sched_getaffinity(0))
    return ProcessPoolExecutor(max_workers=workers or max(1, min(16, cores)), mp_context=mp.get_context("spawn"))


def submit_forest(ex: ProcessPoolExecutor, make: str, arg, n_trees: int, seed: int, max_features, bootstrap: bool,
                  min_samples_split: int = 1):
    """Futures of trees 0..n_trees-1 (collect with [f.result() for f in ...])."""
    return [ex.submit(oracle_tree, make, arg, t, seed, max_features, bootstrap, min_samples_split)
            for t in range(n_trees)]


def tree_digest(left, right, feature, threshold, value) -> str:
    """SHA-256 of a canonical tree's arrays (u32 children, u16 features, f32
    thresholds, u32 leaf classes), so a forest can be pinned in a few bytes."""
    h = hashlib.sha256()
    for a, dt in ((left, np.uint32), (right, np.uint32), (feature, np.uint16), (threshold, np.float32),
                  (value, np.uint32)):
        h.update(np.ascontiguousarray(np.asarray(a).astype(dt)).tobytes())
    return h.hexdigest()


def oracle_digest(t: O.Tree) -> str:
    return tree_digest(t.left, t.right, t.feature, t.threshold, t.value)
