"""CPU oracle for the cudatree_b200 random-forest fit + predict path.

TEST INFRASTRUCTURE ONLY.  Nothing in the shipped package imports this
module; only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg use it, and only as the checker.

What it is
----------
A NumPy restatement of CudaTree's tree-growing algorithm (reference
``cudatree/random_tree.py`` + ``cudatree/cuda_kernels/dfs_module.cu``) with the
launch-shape-dependent parts of the reference replaced by one canonical rule
that the CUDA path must reproduce bit for bit:

* split arithmetic = the reference's DFS form (``dfs_module.cu:348-369`` int64
  sums of squared class counts updated as ``+2*cnt+1`` / ``-2*cnt+1``
  (``dfs_module.cu:392-398``); impurity in fp64 as
  ``(1 - S/(n*n)) * (n/N)`` (``dfs_module.cu:404-407``); candidate positions
  skipped when ``x[p] + 1e-5 >= x[p+1]`` in fp64 (``dfs_module.cu:400``,
  ``common_func.cu:1``); child impurities kept as fp32 (``dfs_module.cu:421``).
* selection: minimum fp64 score ``imp_L + imp_R``; ties go to the lowest
  feature id, then the lowest position (replaces the reference's
  range/thread-order tie-break, ``dfs_module.cu:482``, ``:174-199``).
* feature subset per node: the first ``max_features`` non-constant features of
  a per-node pseudo-random permutation (the reference's BFS kernel skips
  constant features the same way, ``bfs_module.cu:130-140``; its permutation
  is host ``np.random`` state, ``random_tree.py:38-48``).  The permutation is a
  keyed 4-round Feistel network with cycle walking, keyed by a hash of the
  node's root-to-node path, so it does not depend on traversal order.
* bootstrap = the unique set of N draws with replacement
  (``random_forest.py:123-124``); draws come from SplitMix64 streams.
* threshold = fp32 of the fp64 midpoint (``random_tree.py:641-644``).
* leaf value = label of the first row of the leaf in feature 0's sorted order
  (``random_tree.py:50-63``) with a STABLE presort (ties by row index).
* leaf when the parent-reported impurity is exactly 0.0, when
  ``n < min_samples_split`` or when no candidate split exists
  (``random_tree.py:587-634``, ``:113-163``).
* node numbering: breadth-first level order, left child before right child.
* predict: ``x[f] < thr`` goes left (``predict.cu:63``); majority vote with the
  lowest class winning ties (``random_forest.py:358``).

Pinning: the reference cannot run here (Python 2 + PyCUDA + Parakeet, texture
references that nvcc 12.9 rejects).  Its own tests hold no golden vectors;
they hold known-answer "memorize" tests (zero training error with
``bootstrap=False``: ``test/test_digits.py:10-17``, ``test/test_iris.py:7-14``,
``test/test_diabetes_classify.py:7-14``) and accuracy-vs-scikit-learn tests
(``test/helpers.py:4-28``).  ``tests/test_oracle.py`` runs those against this
oracle, and ``reference_dfs_node_split`` below restates the reference's DFS
kernel chain literally so the canonical rule's minimum impurity can be checked
against it node by node.
"""
from __future__ import annotations

import math
from collections import deque
from dataclasses import dataclass, field

import numpy as np

M64 = (1 << 64) - 1
GOLDEN = 0x9E3779B97F4A7C15
DIFF_THRESHOLD = 0.00001  # common_func.cu:1

# Stream separators for the counter-based generator (arbitrary odd constants).
K_TREE = 0x243F6A8885A308D3
K_BOOT = 0x6A09E667F3BCC909
K_ROOT = 0xBB67AE8584CAA73B
K_LEFT = 0xA54FF53A5F1D36F1
K_RIGHT = 0x3C6EF372FE94F82B


# ----------------------------------------------------------------------------
# Counter-based RNG (SplitMix64 output function, Steele/Lea/Flood 2014)
# ----------------------------------------------------------------------------
def mix64(z: int) -> int:
    z &= M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def mix64_np(z: np.ndarray) -> np.ndarray:
    z = z.astype(np.uint64, copy=True)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def tree_key(seed: int, tree: int) -> int:
    return mix64((mix64(seed ^ K_TREE) + (tree + 1) * GOLDEN) & M64)


def root_key(tkey: int) -> int:
    return mix64(tkey ^ K_ROOT)


def child_key(key: int, side: int) -> int:
    return mix64(key ^ (K_RIGHT if side else K_LEFT))


def bootstrap_draws(seed: int, tree: int, n: int) -> np.ndarray:
    """N draws with replacement: row_i = (hi32(splitmix(bk, i)) * N) >> 32."""
    bk = mix64(tree_key(seed, tree) ^ K_BOOT)
    i = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        state = np.uint64(bk) + (i + np.uint64(1)) * np.uint64(GOLDEN)
    u = mix64_np(state)
    hi = u >> np.uint64(32)
    with np.errstate(over="ignore"):
        rows = (hi * np.uint64(n)) >> np.uint64(32)
    return rows.astype(np.int64)


def bootstrap_rows(seed: int, tree: int, n: int, bootstrap: bool) -> np.ndarray:
    """In-bag row set (sorted unique), random_forest.py:113-144."""
    if not bootstrap:
        return np.arange(n, dtype=np.int64)
    return np.unique(bootstrap_draws(seed, tree, n))


def feistel_half_bits(n_features: int) -> int:
    return max(1, ((n_features - 1).bit_length() + 1) // 2)


def feistel(x: int, key: int, h: int) -> int:
    mask = (1 << h) - 1
    left, right = x >> h, x & mask
    for r in range(4):
        fr = mix64((key + ((r << 16) | right) * GOLDEN) & M64) & mask
        left, right = right, left ^ fr
    return (left << h) | right


def feature_perm(i: int, n_features: int, key: int) -> int:
    """i-th feature of the node's permutation (Feistel + cycle walking)."""
    h = feistel_half_bits(n_features)
    x = feistel(i, key, h)
    while x >= n_features:
        x = feistel(x, key, h)
    return x


# ----------------------------------------------------------------------------
# Data preparation (random_forest.py:85-99, :215-248, util.py:40-49)
# ----------------------------------------------------------------------------
def compact_labels(y) -> tuple[np.ndarray, np.ndarray]:
    table = np.unique(np.asarray(y))
    return table, np.searchsorted(table, np.asarray(y)).astype(np.int64)


def index_bytes(n_rows: int) -> int:
    """Reference: smallest uint holding N, uint8 promoted to uint16."""
    return 2 if n_rows <= 0xFFFF else 4


def label_bytes(n_classes: int) -> int:
    return 1 if n_classes <= 0xFF else 2


def presort(x_fm: np.ndarray) -> np.ndarray:
    """Stable ascending argsort per feature row, ties by row index."""
    return np.argsort(x_fm + np.float32(0.0), axis=1, kind="stable")


# ----------------------------------------------------------------------------
# Split scan over one feature's sorted node list (canonical rule)
# ----------------------------------------------------------------------------
@dataclass
class Split:
    score: float
    feature: int
    pos: int
    imp_left: np.float32
    imp_right: np.float32


def scan_sorted(xs: np.ndarray, ls: np.ndarray, totals: np.ndarray):
    """Best (score, pos, impL, impR) over one sorted node list, or None.

    xs: float32 values in sorted order; ls: class ids in the same order;
    totals: int64 class totals of the node.  Follows dfs_module.cu:348-423
    with exact int64 sums and fp64 impurities.
    """
    n = xs.shape[0]
    if n < 2:
        return None
    order = np.argsort(ls, kind="stable")
    sl = ls[order]
    starts = np.searchsorted(sl, np.arange(totals.shape[0]), side="left")
    rank = np.empty(n, dtype=np.int64)
    rank[order] = np.arange(n, dtype=np.int64) - starts[sl]
    dl = 2 * rank + 1
    dr = 1 - 2 * (totals[ls] - rank)
    sum_l = np.cumsum(dl)
    sum_r = int(np.sum(totals * totals)) + np.cumsum(dr)
    x64 = xs.astype(np.float64)
    valid = (x64[:-1] + DIFF_THRESHOLD) < x64[1:]
    if not valid.any():
        return None
    n_left = np.arange(1, n, dtype=np.float64)
    n_right = float(n) - n_left
    imp_l = (1.0 - sum_l[:-1].astype(np.float64) / (n_left * n_left)) * (n_left / float(n))
    imp_r = (1.0 - sum_r[:-1].astype(np.float64) / (n_right * n_right)) * (n_right / float(n))
    score = np.where(valid, imp_l + imp_r, np.inf)
    p = int(np.argmin(score))
    return float(score[p]), p, np.float32(imp_l[p]), np.float32(imp_r[p])


def node_sorted(x_fm: np.ndarray, f: int, members: np.ndarray):
    """Members of a node in feature f's stable sorted order: (order, xs)."""
    xv = x_fm[f, members] + np.float32(0.0)  # -0.0 -> +0.0, as the presort
    order = np.lexsort((members, xv))
    return order, xv[order]


def select_and_split(x_fm, y, members, totals, key, max_features):
    """Feature selection + best split of one node (canonical rule)."""
    n_features = x_fm.shape[0]
    best = None
    taken = 0
    for i in range(n_features):
        f = feature_perm(i, n_features, key)
        xv = x_fm[f, members]
        if xv.min() == xv.max():
            continue
        taken += 1
        order, xs = node_sorted(x_fm, f, members)
        res = scan_sorted(xs, y[members[order]], totals)
        if res is not None:
            score, p, il, ir = res
            if best is None or score < best.score or (score == best.score and f < best.feature):
                best = Split(score, f, p, il, ir)
        if taken == max_features:
            break
    return best


# ----------------------------------------------------------------------------
# Tree growth
# ----------------------------------------------------------------------------
@dataclass
class Tree:
    left: np.ndarray
    right: np.ndarray
    feature: np.ndarray
    threshold: np.ndarray
    value: np.ndarray

    @property
    def n_nodes(self) -> int:
        return int(self.left.shape[0])


def fit_tree(x_fm: np.ndarray, y: np.ndarray, n_classes: int, rows: np.ndarray,
             max_features: int, min_samples_split: int, tkey: int) -> Tree:
    """Grow one fully grown tree over in-bag ``rows``; BFS node order."""
    rows = np.asarray(rows, dtype=np.int64)
    x0 = x_fm[0, rows] + np.float32(0.0)
    members0 = rows[np.lexsort((rows, x0))]  # feature-0 order
    left, right, feat, thr, val = [], [], [], [], []
    queue = deque()

    def new_node():
        left.append(0)
        right.append(0)
        feat.append(0)
        thr.append(np.float32(0.0))
        val.append(0)
        return len(left) - 1

    root = new_node()
    queue.append((root, members0, np.float32(1.0), root_key(tkey)))
    while queue:
        nid, members, imp, key = queue.popleft()
        n = members.shape[0]
        if imp == 0.0 or n < min_samples_split:
            val[nid] = int(y[members[0]])
            continue
        totals = np.bincount(y[members], minlength=n_classes).astype(np.int64)
        best = select_and_split(x_fm, y, members, totals, key, max_features)
        if best is None:
            val[nid] = int(y[members[0]])
            continue
        order, xs = node_sorted(x_fm, best.feature, members)
        a, b = xs[best.pos], xs[best.pos + 1]
        feat[nid] = best.feature
        thr[nid] = np.float32((np.float64(a) + np.float64(b)) / 2.0)
        in_left = np.zeros(n, dtype=bool)
        in_left[order[: best.pos + 1]] = True
        lid, rid = new_node(), new_node()
        left[nid], right[nid] = lid, rid
        queue.append((lid, members[in_left], best.imp_left, child_key(key, 0)))
        queue.append((rid, members[~in_left], best.imp_right, child_key(key, 1)))
    return Tree(np.asarray(left, np.uint32), np.asarray(right, np.uint32),
                np.asarray(feat, np.uint16), np.asarray(thr, np.float32),
                np.asarray(val, np.int64))


@dataclass
class Forest:
    trees: list = field(default_factory=list)
    classes: np.ndarray | None = None
    n_features: int = 0


def fit_forest(x: np.ndarray, y, n_estimators: int = 10, max_features=None,
               bootstrap: bool = True, min_samples_split: int = 1, seed: int = 0) -> Forest:
    x = np.asarray(x, dtype=np.float32)
    classes, yc = compact_labels(y)
    x_fm = np.ascontiguousarray(x.T)
    n, n_features = x.shape
    if max_features is None:
        max_features = int(math.ceil(math.sqrt(n_features)))
    forest = Forest(classes=classes, n_features=n_features)
    for t in range(n_estimators):
        rows = bootstrap_rows(seed, t, n, bootstrap)
        forest.trees.append(fit_tree(x_fm, yc, classes.shape[0], rows, max_features,
                                     min_samples_split, tree_key(seed, t)))
    return forest


# ----------------------------------------------------------------------------
# Predict (predict.cu:50-67, random_forest.py:339-377)
# ----------------------------------------------------------------------------
def tree_predict(tree: Tree, x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.float32)
    idx = np.zeros(x.shape[0], dtype=np.int64)
    rows = np.arange(x.shape[0])
    while True:
        l, r = tree.left[idx], tree.right[idx]
        inner = (l != 0) & (r != 0)
        if not inner.any():
            return tree.value[idx]
        go_left = x[rows, tree.feature[idx].astype(np.int64)] < tree.threshold[idx]
        nxt = np.where(go_left, l, r).astype(np.int64)
        idx = np.where(inner, nxt, idx)


def vote_counts(forest: Forest, x: np.ndarray) -> np.ndarray:
    n_classes = forest.classes.shape[0]
    counts = np.zeros((np.asarray(x).shape[0], n_classes), dtype=np.int64)
    for tree in forest.trees:
        p = tree_predict(tree, x)
        np.add.at(counts, (np.arange(p.shape[0]), p), 1)
    return counts


def predict(forest: Forest, x: np.ndarray) -> np.ndarray:
    return forest.classes[np.argmax(vote_counts(forest, x), axis=1)]


def predict_proba(forest: Forest, x: np.ndarray) -> np.ndarray:
    return vote_counts(forest, x).astype(np.float64) / len(forest.trees)


# ----------------------------------------------------------------------------
# Literal restatement of the reference's DFS split chain, for pinning only
# ----------------------------------------------------------------------------
def reference_dfs_node_split(x_fm, y, lists, n_classes):
    """Restates scan_gini_large/scan_reduce/compute_2d/reduce_2d/find_min_imp.

    ``lists`` holds, for each examined feature in permutation order, the
    node's sorted row indices (reference ``si[f][start:stop]``).  Returns
    ``(imp_left, imp_right, split_pos, feature_slot)`` with the reference's
    float arithmetic (``dfs_module.cu:24-208``, ``random_tree.py:515-578``).
    """
    f32 = np.float32
    n = int(lists[0][1].shape[0])
    n_block = min(int(math.ceil(n / 2000.0)), 50)            # random_tree.py:515-519
    n_range = int(math.ceil(n / float(n_block)))
    threads = 128 if len(y) >= 128 else 32                   # random_forest.py:239-240
    step = threads - 1
    per_feature = []
    for fslot, (f, rows) in enumerate(lists):
        labels = y[rows]
        xs = x_fm[f, rows]
        # scan_gini_large + scan_reduce: cumulative counts before each range
        cum = np.zeros((n_block + 1, n_classes), dtype=np.int64)
        for b in range(n_block):
            lo, hi = b * n_range, min(b * n_range + n_range, n)
            cum[b + 1] = cum[b] + np.bincount(labels[lo:hi], minlength=n_classes)
        total = cum[int(math.ceil(float(n) / n_range))]
        blocks = []
        for b in range(n_block):                              # compute_2d
            count = cum[b].copy()
            ls = int(np.sum(count * count))
            rs = int(np.sum((total - count) ** 2))
            best_l, best_r, best_split = f32(2.0), f32(2.0), 0
            stop_pos = min((b + 1) * n_range, n - 1)
            i = b * n_range
            while i < stop_pos:
                end_pos = step if i + step < stop_pos else stop_pos - i
                for t in range(end_pos):
                    p = i + t
                    c = labels[p]
                    lc = int(count[c])
                    rc = int(total[c]) - lc
                    ls += 2 * lc + 1
                    rs += -2 * rc + 1
                    count[c] += 1
                    if float(xs[p]) + DIFF_THRESHOLD >= float(xs[p + 1]):
                        continue
                    nl = float(p + 1)
                    nr = n - nl
                    il = (1.0 - float(ls) / (nl * nl)) * (nl / n)
                    ir = (1.0 - float(rs) / (nr * nr)) * (nr / n)
                    if il + ir < float(best_r + best_l):
                        best_l, best_r, best_split = f32(il), f32(ir), p
                i += step
            blocks.append((best_l, best_r, best_split))
        min_l, min_r, min_idx = f32(2.0), f32(2.0), 0         # reduce_2d
        for b, (bl, br, _) in enumerate(blocks):
            if min_l + min_r > bl + br:
                min_l, min_r, min_idx = bl, br, b
        per_feature.append((min_l, min_r, blocks[min_idx][2]))
    lanes = []                                                # find_min_imp
    for tid in range(32):
        rl, rr, ridx, rf = f32(2.0), f32(2.0), 0, 0
        for fs in range(tid, len(per_feature), 32):
            l, r, s = per_feature[fs]
            if l + r < rl + rr:
                rl, rr, ridx, rf = l, r, s, fs
        lanes.append((rl + rr, rl, rr, ridx, rf))
    min_imp, min_tid = f32(4.0), 0
    for tid, lane in enumerate(lanes):
        if lane[0] < min_imp:
            min_tid, min_imp = tid, lane[0]
    _, rl, rr, ridx, rf = lanes[min_tid]
    return rl, rr, ridx, rf
