"""Drop-in ``RandomForestClassifier`` for CudaTree's fit/predict path.

Surface of the reference ``cudatree/random_forest.py``:
``RandomForestClassifier(n_estimators=10, max_features=None,
min_samples_split=1, bootstrap=True, verbose=False, debug=False)``
(:45-83), ``fit(samples, target, bfs_threshold=None)`` (:292-336),
``predict(x)`` (:339-362), ``predict_proba(x)`` (:364-377), ``score``
(:379), pickling through ``__reduce__`` (:18-23, :42-43), and the
``fit_init`` / ``fit_release`` pair used by hybrid callers (:215-276).

Everything between the host arrays and the fitted node arrays runs in
``libcudatree_b200.so`` on the current CUDA device; PyTorch only owns the
device buffers and the stream.  Two keyword-only extensions: ``seed`` (the
reference draws from the global ``np.random`` state) and ``fit_mode``
(``"batched"``: all trees of a chunk grow level-synchronously; ``"plain"``:
the reference's per-node depth-first form).  Both give identical trees.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np
import torch

from . import _lib, forest_format, tune_cache
from .forest_format import PACKED_DTYPE
from .random_tree import RandomClassifierTree


def restore_forest(trees, dtype_labels, compt_table=None, n_features=None, params=None):
    """Unpickle hook (reference random_forest.py:18-23).  Unlike the reference,
    the restored forest keeps its label table and can predict."""
    params = dict(params or {})
    f = RandomForestClassifier(params.pop("n_estimators", len(trees)), **params)
    f._trees = list(trees)
    for t in f._trees:
        t.forest = f
    f.dtype_labels = np.dtype(dtype_labels)
    if compt_table is not None:
        f.compt_table = np.asarray(compt_table)
        f.n_labels = int(f.compt_table.shape[0])
    f.n_features = n_features
    return f


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("cudatree_b200 needs a CUDA device (there is no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


PAD_BYTES = 64  # index buffers are read up to 15 bytes past their end by 16-byte bulk copies


def _dev_bytes(nbytes: int, dev) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1) + PAD_BYTES, dtype=torch.uint8, device=dev)


def _to_dev(a: np.ndarray, dev) -> torch.Tensor:
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.uint8).reshape(-1)).to(dev, non_blocking=False)


def best_index_bytes(n_rows: int) -> int:
    """Reference get_best_dtype(n) with uint8 promoted to uint16 (random_forest.py:224-227)."""
    return 2 if n_rows <= 0xFFFF else 4


def default_bfs_threshold(n_labels: int, n_samples: int, max_features: int) -> int:
    """Reference random_forest.py:278-289 ("Titan" regression, clamped)."""
    t = int(4746 + 4 * n_labels + 0.0651 * n_samples - 75 * max_features)
    return max(min(t, 50000), 2000)


def pack_trees(trees):
    """Flatten breadth-first trees into ct_packed_node records + tree offsets."""
    sizes = [t.n_nodes for t in trees]
    offsets = np.zeros(len(trees), dtype=np.uint32)
    if trees:
        offsets[1:] = np.cumsum(sizes[:-1])
    packed = np.zeros(int(sum(sizes)), dtype=PACKED_DTYPE)
    for t, off, n in zip(trees, offsets, sizes):
        sl = packed[int(off):int(off) + n]
        inner = t.left_children != 0
        if np.any(t.right_children[inner] != t.left_children[inner] + 1):
            raise ValueError("tree is not in breadth-first order (right != left + 1)")
        sl["threshold"] = t.feature_threshold_array
        sl["feature"] = t.feature_idx_array
        sl["left"] = t.left_children
        sl["value"] = t.values_array
    return packed, offsets




def compact_labels(y):
    """(table, ids): the sorted distinct labels and each label's index in the
    table, as np.unique(y, return_inverse=True) gives them (the reference's
    __compact_labels, random_forest.py:85-99).  Integer labels of modest
    range take a counting path (linear, no sort)."""
    y = np.asarray(y)
    if y.dtype.kind in "iu" and y.size:
        lo, hi = int(y.min()), int(y.max())
        if hi - lo < (1 << 22) and -(1 << 62) < lo and hi < (1 << 62):
            off = y if lo == 0 else y.astype(np.int64) - lo
            present = np.bincount(off, minlength=hi - lo + 1) > 0
            table = (np.flatnonzero(present) + lo).astype(y.dtype)
            # ids in the narrowest unsigned type (the label width of the fit)
            dt = np.uint8 if table.size <= 0x100 else np.uint16 if table.size <= 0x10000 else np.int64
            lut = (np.cumsum(present, dtype=np.int64) - 1).astype(dt)
            return table, lut[off]
    return np.unique(y, return_inverse=True)


def fetch_tree_columns(tb, n_nodes, kk, dev):
    """(node counts, [left, right, feature, threshold, value]) of the trees in
    slots 0..kk-1 of raw tree buffers, canonical order, concatenated (one
    device canonicalization and one read-back)."""
    counts = n_nodes[:kk].cpu().numpy().astype(np.uint32)
    total = int(counts.sum())
    cols = [np.empty(total, dt) for dt in (np.uint32, np.uint32, np.uint16, np.float32, np.uint32)]
    sb = int(_lib.load().ct_fetch_trees_scratch(total, kk))
    scratch = _dev_bytes(sb, dev)
    _lib.call("ct_fetch_trees", C.byref(tb), kk, counts.ctypes.data, _ptr(scratch), sb,
              *[c.ctypes.data for c in cols], _stream())
    return counts, cols


def unpack_trees(packed, offsets, n_features, dtype_labels):
    """Inverse of pack_trees: RandomClassifierTree objects from packed nodes."""
    from .random_tree import restore_tree
    packed = np.asarray(packed, dtype=PACKED_DTYPE)
    offsets = np.asarray(offsets, dtype=np.int64)
    ends = np.append(offsets[1:], packed.shape[0])
    dt = np.dtype(dtype_labels)
    trees = []
    for o, e in zip(offsets.tolist(), ends.tolist()):
        sl = packed[o:e]
        left = sl["left"].astype(np.uint32)
        right = np.where(left != 0, left + 1, 0).astype(np.uint32)
        trees.append(restore_tree(left, right, sl["threshold"].astype(np.float32), sl["value"].astype(dt),
                                  sl["feature"].astype(np.uint16), dt.str, n_features))
    return trees


def _predict_packed(packed, offsets, n_trees, x, n_features, n_classes, want_votes, compact=False):
    """Walk the forest on the device: packed nodes (ct_predict) or, with
    compact=True, a device tensor of 8-byte compact nodes (ct_predict_compact).
    The library checks the forest before it walks it."""
    dev = _device()
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    if x.ndim != 2 or x.shape[1] != n_features:
        raise ValueError(f"x must have shape [n, {n_features}]")
    n = x.shape[0]
    if n == 0:
        return np.zeros((0, n_classes) if want_votes else (0,), dtype=np.uint32)
    nodes = packed if isinstance(packed, torch.Tensor) else _to_dev(packed, dev)
    offs = offsets if isinstance(offsets, torch.Tensor) else _to_dev(offsets.astype(np.uint32), dev)
    xd = torch.from_numpy(x).to(dev)
    votes = torch.empty((n, n_classes), dtype=torch.int32, device=dev)  # also the tree-group vote table
    pred = torch.empty((n,), dtype=torch.int32, device=dev)
    n_nodes = nodes.numel() * nodes.element_size() // (8 if compact else 16)
    _lib.call("ct_predict_compact" if compact else "ct_predict", _ptr(nodes), n_nodes, _ptr(offs), n_trees, _ptr(xd),
              n, n_features, n_classes, _ptr(votes), _ptr(pred), _stream())
    return (votes if want_votes else pred).cpu().numpy().view(np.uint32)


class RandomForestClassifier:
    """A random forest classifier (Gini, fully grown trees) on one B200."""

    def __init__(self, n_estimators=10, max_features=None, min_samples_split=1, bootstrap=True,
                 verbose=False, debug=False, *, seed=None, fit_mode="batched", subtree_cutoff=32,
                 autotune=False):
        if fit_mode not in ("batched", "plain"):
            raise ValueError("fit_mode must be 'batched' or 'plain'")
        if not 0 <= int(subtree_cutoff) <= 128:
            raise ValueError("subtree_cutoff must be in [0, 128]")
        # nodes of at most subtree_cutoff rows are grown whole by one warp
        # (same trees; 0 keeps every node in the level steps)
        self.subtree_cutoff = int(subtree_cutoff)
        # time candidate fit options on a few trees before the first fit of a
        # data shape (options never change the trees, only the speed)
        self.autotune_fit = bool(autotune)
        self._tuned = None
        self.n_estimators = int(n_estimators)
        self.max_features = max_features
        self.min_samples_split = int(min_samples_split)
        self.bootstrap = bool(bootstrap)
        self.verbose = verbose
        self.debug = debug
        self.seed = seed
        self.fit_mode = fit_mode
        self._trees = []
        self._packed = None
        self.last_fit_timing = {}
        self.last_fit_stats = None
        self.profile = False  # record CUDA-event time per kernel group
        # batched form: run the levels from the host (one round trip per
        # level) instead of as one CUDA graph with a device-side loop
        self.host_level_loop = False
        # nodes per level step (0: 2^20); a wider level takes several steps
        self.step_nodes = 0
        # keep no index lists for two-valued features (one row-order list per
        # node and a value bit per row stand for them); False keeps them all
        self.virtual_features = True
        # batched form: levels of at most this many samples run in the loop
        # graph, larger ones from the host (0 or 0xffffffff: all of them)
        self.graph_samples = 0

    # ------------------------------------------------------------ pickling
    def _params(self):
        return dict(n_estimators=self.n_estimators, max_features=self.max_features,
                    min_samples_split=self.min_samples_split,
                    bootstrap=self.bootstrap, seed=self.seed, fit_mode=self.fit_mode,
                    subtree_cutoff=self.subtree_cutoff)

    def __reduce__(self):
        """A fitted forest pickles as its flat format (forest_format); an
        unfitted one as its constructor arguments."""
        if self._trees:
            return forest_format.restore_forest_flat, (forest_format.dumps(self),)
        return restore_forest, (self._trees, getattr(self, "dtype_labels", np.dtype(np.uint8)).str,
                                getattr(self, "compt_table", None), getattr(self, "n_features", None),
                                self._params())

    def to_bytes(self) -> bytes:
        """The fitted forest in the versioned flat format (forest_format)."""
        return forest_format.dumps(self)

    @classmethod
    def from_bytes(cls, data: bytes) -> "RandomForestClassifier":
        """A forest stored by to_bytes or save; ValueError when the bytes are
        not a valid flat forest."""
        return forest_format.loads(data)

    def save(self, path) -> None:
        forest_format.save(self, path)

    @classmethod
    def load(cls, path) -> "RandomForestClassifier":
        return forest_format.load(path)

    # ------------------------------------------------------------- fitting
    def fit_init(self, samples, target):
        """Validate, compact labels, upload and presort (random_forest.py:215-266)."""
        x_src = samples if isinstance(samples, torch.Tensor) else None
        x = samples.numpy() if isinstance(samples, torch.Tensor) else np.asarray(samples)
        y = target.numpy() if isinstance(target, torch.Tensor) else np.asarray(target)
        if x.ndim != 2:
            raise ValueError("samples must be a 2-D array [n_samples, n_features]")
        if y.ndim != 1 or y.shape[0] != x.shape[0]:
            raise ValueError("target must be a 1-D array with one label per sample")
        if x.shape[0] == 0:
            raise ValueError("cannot fit on zero samples")
        x32 = np.ascontiguousarray(x, dtype=np.float32)
        self.samples, self.target = samples, target  # as the reference keeps them (random_forest.py:215-266)
        self._next_tree = 0
        self.compt_table, y_c = compact_labels(y)
        self.n_labels = int(self.compt_table.shape[0])
        if self.n_labels > _lib.MAX_CLASSES:
            raise ValueError(f"at most {_lib.MAX_CLASSES} classes are supported")
        self.n_samples, self.n_features = x32.shape
        if self.n_features > _lib.MAX_FEATURES - 1:
            raise ValueError("too many features")
        self.stride = self.n_samples
        self.index_bytes = best_index_bytes(self.n_samples)
        self.dtype_indices = np.dtype(np.uint16 if self.index_bytes == 2 else np.uint32)
        self.dtype_labels = np.dtype(np.uint8 if self.n_labels <= 0xFF else np.uint16)
        m = self.max_features
        if m is None:
            m = int(math.ceil(math.sqrt(self.n_features)))
        m = int(m)
        if not (0 < m <= self.n_features):
            raise ValueError("max_features must be in [1, n_features]")
        self._m = m
        self.bfs_threshold = default_bfs_threshold(self.n_labels, self.n_samples, m)
        self._seed = int(np.random.randint(0, 2**62)) if self.seed is None else int(self.seed)
        dev = _device()
        t0 = time.perf_counter()
        if x_src is not None and x_src.dtype == torch.float32 and x_src.is_contiguous():
            xd = x_src.to(dev, non_blocking=True)  # pinned host tensors copy asynchronously
        else:
            xd = torch.from_numpy(x32).to(dev)
        self._x_fm = torch.empty((self.n_features, self.n_samples), dtype=torch.float32, device=dev)
        nan = torch.zeros(1, dtype=torch.int32, device=dev)
        _lib.call("ct_transpose_rows", _ptr(xd), self.n_samples, self.n_features, _ptr(self._x_fm), _ptr(nan),
                  _stream())
        self._labels = _to_dev(y_c.astype(self.dtype_labels), dev)
        self._presort = _dev_bytes(self.n_features * self.n_samples * self.index_bytes, dev)
        ws = C.c_size_t()
        _lib.call("ct_presort_workspace_size", self.n_samples, self.n_features, C.byref(ws))
        pws = _dev_bytes(ws.value, dev)
        _lib.call("ct_presort", _ptr(self._x_fm), self.n_samples, self.n_features, self.index_bytes,
                  _ptr(self._presort), _ptr(pws), ws.value, _stream())
        del pws
        if int(nan.item()):
            self.fit_release()
            raise ValueError("samples contain NaN")
        self.last_fit_timing = {"upload_presort_s": time.perf_counter() - t0}

    def _problem(self) -> _lib.Problem:
        return _lib.Problem(_ptr(self._x_fm), _ptr(self._labels), _ptr(self._presort), self.n_samples,
                            self.n_features, self.n_labels, self.index_bytes, self.dtype_labels.itemsize,
                            self._m, self.min_samples_split, int(self.bootstrap), self._seed)

    @property
    def sorted_indices(self):
        """The device presort [F][N] (row ids in each feature's value order)."""
        return getattr(self, "_presort", None)

    def _get_sorted_indices(self, sorted_indices):
        """(tree index, rows) for the next tree of a per-tree loop
        (random_forest.py:113-144, called by hybridforest/builder.py:131).
        The bootstrap sample is drawn inside the tree's fit from the forest's
        seed and this index, so a per-tree loop grows the same trees as fit()."""
        t = self._next_tree
        self._next_tree += 1
        return t, self.n_samples

    def fit_release(self):
        self._x_fm = None
        self._labels = None
        self._presort = None

    def _slot_bytes(self) -> int:
        n, f = self.n_samples, self.n_features
        return 2 * f * n * self.index_bytes + n + 2 * n * 20

    def trees_in_flight(self, mode: str, query_free: bool = False) -> int:
        """Trees grown by one batched call: all of them when their lists and
        workspace take at most half of the device, else as many as fit in 70 %
        of the free memory.  The free-memory query is skipped when the forest
        is small against the device: it took 1-77 ms per call on B200."""
        if mode == "plain":
            return 1
        prob = self._problem()
        opts = self._fit_options(_lib.CT_FIT_BATCHED, 0)

        def need(k):
            ws = C.c_size_t()
            _lib.call("ct_fit_workspace_size", C.byref(prob), k, C.byref(opts), C.byref(ws))
            return k * self._slot_bytes() + ws.value

        k = self.n_estimators
        total = torch.cuda.get_device_properties(_device()).total_memory
        if not query_free and need(k) <= total // 2:
            return k
        free, _ = torch.cuda.mem_get_info()
        budget = int(free * 0.7)
        while k > 1 and need(k) > budget:
            k = max(1, k // 2)
        return k

    def _fit_trees(self, first: int, count: int, mode: str, bfs_threshold: int):
        try:
            return self._fit_trees_k(first, count, mode, bfs_threshold, self.trees_in_flight(mode))
        except torch.OutOfMemoryError:  # another tenant holds memory: size the batch from the free memory
            torch.cuda.empty_cache()
            return self._fit_trees_k(first, count, mode, bfs_threshold, self.trees_in_flight(mode, query_free=True))

    def _fit_trees_k(self, first: int, count: int, mode: str, bfs_threshold: int, in_flight: int):
        dev = _device()
        prob = self._problem()
        n, f = self.n_samples, self.n_features
        mode_id = _lib.CT_FIT_PLAIN if mode == "plain" else _lib.CT_FIT_BATCHED
        k = min(in_flight, count)
        slots = 1 if mode == "plain" else k
        per_call = 1 if mode == "plain" else k
        si0 = _dev_bytes(slots * f * n * self.index_bytes, dev)
        si1 = _dev_bytes(slots * f * n * self.index_bytes, dev)
        mark = _dev_bytes(_lib.mark_bytes(n, slots), dev)
        lists = _lib.Lists(_ptr(si0), _ptr(si1), _ptr(mark), n, slots)
        cap = 2 * n
        raw = {name: torch.empty(per_call * cap, dtype=torch.int32, device=dev)
               for name in ("left", "right", "feature", "threshold", "value")}
        n_nodes = torch.zeros(per_call, dtype=torch.int32, device=dev)
        tb = _lib.TreeBuffers(_ptr(raw["left"]), _ptr(raw["right"]), _ptr(raw["feature"]),
                              _ptr(raw["threshold"]), _ptr(raw["value"]), _ptr(n_nodes), cap)
        opts = self._fit_options(mode_id, bfs_threshold)
        opts.flags |= (_lib.CT_FIT_PROFILE if self.profile else 0) | (_lib.CT_FIT_HOST_LOOP if self.host_level_loop else 0)
        ws = C.c_size_t()
        _lib.call("ct_fit_workspace_size", C.byref(prob), per_call, C.byref(opts), C.byref(ws))
        work = _dev_bytes(ws.value, dev)
        trees = []
        stats = None
        for t0 in range(first, first + count, per_call):
            kk = min(per_call, first + count - t0)
            _lib.call("ct_fit", C.byref(prob), C.byref(lists), t0, kk, C.byref(opts), C.byref(tb),
                      _ptr(work), ws.value, _stream())
            st = _lib.fit_stats()
            if stats is None:
                stats = st
            else:
                for key in ("launches", "ms", "bytes"):
                    stats[key] = [a + b for a, b in zip(stats[key], st[key])]
                stats["steps"] += st["steps"]
                stats["total_launches"] += st["total_launches"]
            trees.extend(self._fetch_trees(tb, n_nodes, kk, dev))
        self.last_fit_stats = stats
        return trees

    def _fetch_trees(self, tb, n_nodes, kk, dev):
        """The kk trees of the last ct_fit call, canonical order, as tree objects
        over slices of five concatenated host arrays (one read-back)."""
        counts, cols = fetch_tree_columns(tb, n_nodes, kk, dev)
        out, o = [], 0
        for c in counts.tolist():
            out.append(self._make_tree(*[col[o:o + c] for col in cols]))
            o += c
        return out

    def _make_tree(self, left, right, feat, thr, val):
        tree = RandomClassifierTree(self)
        tree.left_children = left
        tree.right_children = right
        tree.feature_idx_array = feat
        tree.feature_threshold_array = thr
        tree.values_array = val.astype(self.dtype_labels)
        tree.dtype_labels = self.dtype_labels
        tree.n_features = self.n_features
        return tree

    def fit(self, samples, target, bfs_threshold=None):
        """Grow n_estimators trees (reference random_forest.py:292-336); returns self."""
        t0 = time.perf_counter()
        self.fit_init(samples, target)
        if bfs_threshold is not None:
            self.bfs_threshold = int(bfs_threshold)
        if self.autotune_fit and self._tuned is None:
            self._tuned = tune_cache.get(self._tune_key(self.fit_mode))
            if self._tuned is None:
                self._run_autotune(self.fit_mode, min(8, self.n_estimators))
            if bfs_threshold is None and self.fit_mode == "plain":
                self.bfs_threshold = self._tuned["bfs_threshold"]
        if self.verbose:
            print(f"bfs_threshold : {self.bfs_threshold}; bootstrap : {self.bootstrap}; "
                  f"min_samples_split : {self.min_samples_split}; fit_mode : {self.fit_mode}")
            print(f"n_samples : {self.n_samples}; n_features : {self.n_features}; "
                  f"n_labels : {self.n_labels}; max_features : {self._m}")
        self._trees = self._fit_trees(0, self.n_estimators, self.fit_mode, self.bfs_threshold)
        self._packed = None
        self.fit_release()
        torch.cuda.synchronize()
        self.last_fit_timing["fit_s"] = time.perf_counter() - t0
        return self

    # ---------------------------------------------------------- autotune
    def _fit_options(self, mode_id, bfs_threshold):
        t = self._tuned or {}
        o = _lib.FitOptions(mode_id, int(bfs_threshold), int(t.get("subtree_cutoff", self.subtree_cutoff)),
                            int(t.get("scan_piece", 0)))
        if not self.virtual_features:
            o.flags |= _lib.CT_FIT_NO_VIRTUAL
        o.step_nodes = int(self.step_nodes)
        o.graph_samples = int(self.graph_samples)
        o.part_shape = int(t.get("part_shape", 0))
        o.huge_rows = int(t.get("huge_rows", 0))
        o.small_rows = int(t.get("small_rows", 0))
        return o

    def _shape_key(self, mode):
        return (mode, self.n_samples, self.n_features, self.n_labels, self._m, self.index_bytes,
                bool(self.bootstrap), self.min_samples_split)

    def _tune_key(self, mode):
        return tune_cache.key(torch.cuda.get_device_name(_device()), self._shape_key(mode))

    def _run_autotune(self, mode, sample_trees):
        dev = _device()
        prob = self._problem()
        n, f = self.n_samples, self.n_features
        mode_id = _lib.CT_FIT_PLAIN if mode == "plain" else _lib.CT_FIT_BATCHED
        slots = 1 if mode == "plain" else sample_trees
        si0 = _dev_bytes(slots * f * n * self.index_bytes, dev)
        si1 = _dev_bytes(slots * f * n * self.index_bytes, dev)
        mark = _dev_bytes(_lib.mark_bytes(n, slots), dev)
        lists = _lib.Lists(_ptr(si0), _ptr(si1), _ptr(mark), n, slots)
        cap = 2 * n
        raw = [torch.empty(sample_trees * cap, dtype=torch.int32, device=dev) for _ in range(5)]
        n_nodes = torch.zeros(sample_trees, dtype=torch.int32, device=dev)
        tb = _lib.TreeBuffers(*[_ptr(r) for r in raw], _ptr(n_nodes), cap)
        wsb = C.c_size_t()
        _lib.call("ct_autotune_workspace_size", C.byref(prob), sample_trees, mode_id, C.byref(wsb))
        work = _dev_bytes(wsb.value, dev)
        best = _lib.FitOptions()
        ms = C.c_float()
        _lib.call("ct_autotune", C.byref(prob), C.byref(lists), sample_trees, mode_id, C.byref(tb), _ptr(work),
                  wsb.value, C.byref(best), C.byref(ms), _stream())
        self._tuned = {"scan_piece": int(best.scan_piece), "subtree_cutoff": int(best.subtree_cutoff),
                       "bfs_threshold": int(best.bfs_threshold) or self.bfs_threshold,
                       "part_shape": int(best.part_shape), "huge_rows": int(best.huge_rows),
                       "small_rows": int(best.small_rows),
                       "sample_trees": sample_trees, "sample_ms": float(ms.value)}
        tune_cache.put(self._tune_key(mode), self._tuned)
        return self._tuned

    def autotune(self, samples, target, sample_trees=8):
        """Choose fit options for this data shape by timing candidate fits of
        sample_trees trees (the reference's offline threshold estimate,
        estimate_threshold.py, done on the device at hand); later fits of the
        same shape with autotune=True reuse the choice, in this process and,
        through tune_cache's file, in later ones.  Returns it."""
        self.fit_init(samples, target)
        try:
            return dict(self._run_autotune(self.fit_mode, max(1, min(int(sample_trees), self.n_estimators))))
        finally:
            self.fit_release()

    # ----------------------------------------------------------- predict
    def _device_forest(self, compact=None):
        """(nodes, tree offsets, is_compact) on the device.  compact=None picks
        the 8-byte compact form whenever the trees fit it."""
        if compact is None:
            compact = self._compact_fits()
        key = "compact" if compact else "packed"
        if self._packed is None:
            self._packed = {}
        if key not in self._packed:
            dev = _device()
            packed, offsets = pack_trees(self._trees)
            nodes, offs = _to_dev(packed, dev), _to_dev(offsets, dev)
            if compact:
                out = torch.empty(packed.shape[0] * 8, dtype=torch.uint8, device=dev)
                _lib.call("ct_compact_forest", _ptr(nodes), packed.shape[0], self.n_features,
                          max(t.n_nodes for t in self._trees), _ptr(out), _stream())
                nodes = out
            self._packed[key] = (nodes, offs, compact)
        return self._packed[key]

    def _compact_fits(self) -> bool:
        most = max(t.n_nodes for t in self._trees)
        return bool(_lib.load().ct_compact_fits(self.n_features, most))

    def _votes(self, x, compact=None) -> np.ndarray:
        if not self._trees:
            raise ValueError("forest is not fitted")
        nodes, offs, cp = self._device_forest(compact)
        return _predict_packed(nodes, offs, len(self._trees), x, self.n_features, self.n_labels, True, cp)

    def predict(self, x):
        """Majority vote, lowest class on ties, in original label space (random_forest.py:339-362)."""
        if not self._trees:
            raise ValueError("forest is not fitted")
        nodes, offs, cp = self._device_forest()
        res = _predict_packed(nodes, offs, len(self._trees), x, self.n_features, self.n_labels, False, cp)
        return self.compt_table[res.astype(np.int64)]

    def predict_proba(self, x):
        """Vote fractions per class, float64 [n, n_labels] (random_forest.py:364-377)."""
        return self._votes(x).astype(np.float64) / len(self._trees)

    def score(self, X, Y):
        return float(np.mean(self.predict(X) == np.asarray(Y)))
