"""CPU-side checks of the C ABI: the library loads, exports every symbol the
header declares, validates arguments without touching a GPU, and the
host-side canonical renumbering matches a breadth-first walk."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from cudatree_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "cudatree_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ct_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_header_symbols():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 14
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.PROTOTYPES), "ctypes prototypes missing for some exports"
    assert "sm_100a" in _lib.version()


def test_struct_layouts_match_header_sizes():
    assert C.sizeof(_lib.Node) == 32
    assert C.sizeof(_lib.SplitResult) == 32
    assert C.sizeof(_lib.PackedNode) == 16
    from cudatree_b200 import serving
    assert C.sizeof(serving.ServerConfig) == 48
    assert C.sizeof(serving.Request) == 96
    assert C.sizeof(serving.ServerStats) == 152
    assert np.dtype(_lib.NODE_DTYPE_FIELDS).itemsize == 32
    assert np.dtype(_lib.SPLIT_DTYPE_FIELDS).itemsize == 32


def test_argument_errors_are_reported_without_gpu():
    lib = _lib.load()
    st = lib.ct_predict(None, 0, None, 0, None, 0, 0, 0, None, None, None)
    assert st == 1
    assert "NULL" in _lib.last_error()
    prob = _lib.Problem(1, 1, 1, 10, 4, 3, 3, 1, 9, 1, 0, 0)  # uint16 index width is 2 or 4 only
    ws = C.c_size_t()
    st = lib.ct_fit(C.byref(prob), None, 0, 1, None, None, None, 0, None)
    assert st != 0
    with pytest.raises(_lib.CudaTreeError):
        _lib.check(st)


def test_workspace_size_queries_are_host_only():
    prob = _lib.Problem(1, 1, 1, 581012, 54, 7, 4, 1, 7, 1, 1, 0)
    ws = C.c_size_t()
    for mode in (_lib.CT_FIT_PLAIN, _lib.CT_FIT_BATCHED):
        opts = _lib.FitOptions(mode, 0, 0, 0)
        _lib.call("ct_fit_workspace_size", C.byref(prob), 8, C.byref(opts), C.byref(ws))
        assert ws.value > 0
    _lib.call("ct_split_workspace_size", C.byref(prob), 100, 1 << 20, C.byref(ws))
    assert ws.value > 0
    _lib.call("ct_presort_workspace_size", 1000, 10, C.byref(ws))
    assert ws.value >= 4 * 4 * 1000 * 10


def _random_raw_tree(rng, n_inner):
    # grow a random binary tree with ids in random allocation order
    n = 2 * n_inner + 1
    perm = np.concatenate([[0], 1 + rng.permutation(n - 1)])
    left = np.zeros(n, np.uint32)
    right = np.zeros(n, np.uint32)
    feat = np.zeros(n, np.uint32)
    thr = np.zeros(n, np.float32)
    val = rng.integers(0, 5, n).astype(np.uint32)
    leaves = [0]
    nxt = 1
    for _ in range(n_inner):
        k = int(rng.integers(0, len(leaves)))
        v = leaves.pop(k)
        a, b = perm[nxt], perm[nxt + 1]
        nxt += 2
        left[perm[v] if False else v] = a
        right[v] = b
        feat[v] = rng.integers(0, 50)
        thr[v] = rng.normal()
        val[v] = 0
        leaves += [a, b]
    return left, right, feat, thr, val


def test_canonicalize_is_breadth_first():
    rng = np.random.default_rng(0)
    left, right, feat, thr, val = _random_raw_tree(rng, 200)
    n = left.shape[0]
    out = [np.empty(n, np.uint32), np.empty(n, np.uint32), np.empty(n, np.uint16), np.empty(n, np.float32),
           np.empty(n, np.uint32)]
    _lib.call("ct_tree_canonicalize", left.ctypes.data, right.ctypes.data, feat.ctypes.data, thr.ctypes.data,
              val.ctypes.data, n, *[o.ctypes.data for o in out])
    ol, orr, of, ot, ov = out
    # Python BFS
    order, q = [], [0]
    while q:
        r = q.pop(0)
        order.append(r)
        if left[r] and right[r]:
            q += [int(left[r]), int(right[r])]
    new = {r: i for i, r in enumerate(order)}
    for i, r in enumerate(order):
        inner = left[r] != 0
        assert ol[i] == (new[int(left[r])] if inner else 0)
        assert orr[i] == (new[int(right[r])] if inner else 0)
        assert of[i] == feat[r] and ot[i] == thr[r] and ov[i] == val[r]
    inner = ol != 0
    assert np.all(orr[inner] == ol[inner] + 1)


def test_canonicalize_rejects_unreachable_nodes():
    left = np.array([1, 0, 0, 0], np.uint32)
    right = np.array([2, 0, 0, 0], np.uint32)
    z = np.zeros(4, np.uint32)
    out = [np.empty(4, t) for t in (np.uint32, np.uint32, np.uint16, np.float32, np.uint32)]
    st = _lib.load().ct_tree_canonicalize(left.ctypes.data, right.ctypes.data, z.ctypes.data,
                                         np.zeros(4, np.float32).ctypes.data, z.ctypes.data, 4,
                                         *[o.ctypes.data for o in out])
    assert st == 6 and "unreachable" in _lib.last_error()


def test_compact_fit_rule():
    """Compact nodes hold left << b | feature in 32 bits, b = feature bits."""
    lib = _lib.load()
    assert lib.ct_compact_fits(54, 1 << 26) == 1      # b = 6
    assert lib.ct_compact_fits(54, (1 << 26) + 1) == 0
    assert lib.ct_compact_fits(64, 1 << 26) == 1      # 64 features still need only 6 bits
    assert lib.ct_compact_fits(65, 1 << 26) == 0      # b = 7
    assert lib.ct_compact_fits(1, 1 << 31) == 1       # b = 1
    assert lib.ct_compact_fits(3000, 1 << 20) == 1    # b = 12
    assert lib.ct_compact_fits(0, 10) == 0


def test_compact_labels_matches_np_unique():
    """Label compaction (the reference's __compact_labels) gives exactly the
    table and ids of np.unique(return_inverse=True), on its counting path and
    its sorting path."""
    from cudatree_b200.random_forest import compact_labels
    rng = np.random.default_rng(0)
    cases = [rng.integers(-5, 40, 1000), rng.integers(0, 7, 5000).astype(np.uint8), np.array([3, 3, 3]),
             rng.integers(0, 2**40, 100), rng.normal(size=50), np.array(["b", "a", "b"]),
             rng.integers(0, 3, 10).astype(np.uint64), np.array([2**63 + 5, 2**63 + 1], dtype=np.uint64)]
    for y in cases:
        t, i = compact_labels(y)
        t2, i2 = np.unique(y, return_inverse=True)
        assert t.dtype == t2.dtype
        np.testing.assert_array_equal(t, t2)
        np.testing.assert_array_equal(i, i2)


def _check(packed, offsets, n_features=4, n_classes=3):
    packed = np.ascontiguousarray(packed)
    offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
    return _lib.load().ct_check_forest(packed.ctypes.data, packed.shape[0], offsets.ctypes.data,
                                       offsets.shape[0], n_features, n_classes)


def _forest():
    """Two breadth-first trees: a stump (3 nodes) and a depth-2 tree (5 nodes)."""
    from cudatree_b200.random_forest import PACKED_DTYPE
    p = np.zeros(8, dtype=PACKED_DTYPE)
    p["left"] = [1, 0, 0, 1, 3, 0, 0, 0]
    p["feature"] = [2, 0, 0, 0, 3, 0, 0, 0]
    p["value"] = [0, 1, 2, 0, 0, 2, 0, 1]
    return p, np.array([0, 3], np.uint32)


@pytest.mark.parametrize("case", ["ok", "cycle", "self_loop", "child_past_tree", "bad_feature", "bad_class",
                                  "offsets_out_of_order", "offset_past_end"])
def test_malformed_forests_are_rejected_before_any_walk(case):
    """The forest check that ct_predict runs on the device and
    ct_server_add_forest runs on the host, through ct_check_forest: children
    must come after their node inside its tree (so every walk ends), features
    and leaf classes must be in range, tree offsets strictly increasing."""
    p, off = _forest()
    if case == "cycle":
        p["left"][4] = 1  # node 4 of tree 1 points back to its grandparent
    elif case == "self_loop":
        p["left"][3] = 0 + 0  # root becomes a leaf: still valid ...
        p["left"][4] = 1  # ... and node 1 (local) points to itself
    elif case == "child_past_tree":
        p["left"][0] = 2  # right child would be node 3: the next tree's root
    elif case == "bad_feature":
        p["feature"][4] = 4
    elif case == "bad_class":
        p["value"][7] = 3
    elif case == "offsets_out_of_order":
        off = np.array([3, 0], np.uint32)
    elif case == "offset_past_end":
        off = np.array([0, 8], np.uint32)
    st = _check(p, off)
    if case == "ok":
        assert st == 0, _lib.last_error()
    else:
        assert st == 1, case
        assert "malformed forest" in _lib.last_error()


def test_fit_rejects_bad_partition_options_before_any_launch():
    """part_shape beyond CT_PART_SHAPES and huge_rows below 4,096 are refused
    with CT_ERR_ARG before the fit touches the device (the pointers here are
    never dereferenced)."""
    lib = _lib.load()
    fake = 256
    prob = _lib.Problem(fake, fake, fake, 1000, 8, 3, 4, 1, 3, 1, 1, 0)
    lists = _lib.Lists(fake, fake, fake, 1000, 4)
    trees = _lib.TreeBuffers(fake, fake, fake, fake, fake, fake, 2000)
    for shape, huge, small, text in ((4, 0, 0, "part_shape"), (0, 100, 0, "huge_rows"), (0, 0, 100, "small_rows")):
        opts = _lib.FitOptions(_lib.CT_FIT_BATCHED, 0, 0, 0)
        opts.part_shape, opts.huge_rows, opts.small_rows = shape, huge, small
        st = lib.ct_fit(C.byref(prob), C.byref(lists), 0, 4, C.byref(opts), C.byref(trees), C.c_void_p(fake), 0,
                        None)
        assert st == 1 and text in _lib.last_error()


def test_queue_fit_checks_jobs_before_any_launch():
    """ct_fit_queue refuses, with CT_ERR_ARG and no device work, jobs of
    different index widths, a job without trees and tree buffers too small
    for a job (the pointers here are never dereferenced)."""
    lib = _lib.load()
    fake = 256
    jobs = (_lib.FitJob * 2)()
    for k in range(2):
        jobs[k].problem = _lib.Problem(fake, fake, fake, 1000, 8, 3, 2, 1, 3, 1, 1, k)
        jobs[k].lists = _lib.Lists(fake, fake, fake, 1000, 4)
        jobs[k].n_trees = 4
    trees = _lib.TreeBuffers(fake, fake, fake, fake, fake, fake, 2000)
    opts = _lib.FitOptions(_lib.CT_FIT_BATCHED, 0, 0, 0)
    ws = C.c_size_t()
    assert lib.ct_fit_queue_workspace_size(jobs, 2, C.byref(opts), C.byref(ws)) == 0 and ws.value > 0
    jobs[1].problem.index_bytes = 4
    st = lib.ct_fit_queue(jobs, 2, C.byref(opts), C.byref(trees), C.c_void_p(fake), ws.value, None)
    assert st == 1 and "index_bytes" in _lib.last_error()
    jobs[1].problem.index_bytes = 2
    jobs[1].n_trees = 0
    st = lib.ct_fit_queue(jobs, 2, C.byref(opts), C.byref(trees), C.c_void_p(fake), ws.value, None)
    assert st == 1 and "no trees" in _lib.last_error()
    jobs[1].n_trees = 4
    small = _lib.TreeBuffers(fake, fake, fake, fake, fake, fake, 100)
    st = lib.ct_fit_queue(jobs, 2, C.byref(opts), C.byref(small), C.c_void_p(fake), ws.value, None)
    assert st == 1 and "capacity" in _lib.last_error()
    plain = _lib.FitOptions(_lib.CT_FIT_PLAIN, 0, 0, 0)
    st = lib.ct_fit_queue(jobs, 2, C.byref(plain), C.byref(trees), C.c_void_p(fake), ws.value, None)
    assert st == 1 and "batched" in _lib.last_error()
