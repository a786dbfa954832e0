"""Kernel-level parity through the C ABI: presort, bootstrap compaction,
split scan + min-impurity reduction, stable partition.  Bit-exact against the
CPU oracle (integer/index results exact; fp64 scores compared with ==)."""
import ctypes as C

import numpy as np
import pytest

from cudatree_b200 import _lib
from oracle import cudatree_oracle as O

from . import gpu_utils as G

pytestmark = pytest.mark.gpu


def _data(n, f, c, seed, integer=True):
    rng = np.random.default_rng(seed)
    if integer:
        x = rng.integers(0, 6, size=(n, f)).astype(np.float32)
    else:
        x = rng.normal(size=(n, f)).astype(np.float32)
    y = rng.integers(0, c, size=n)
    return x, y


@pytest.mark.parametrize("index_bytes", [2, 4])
def test_presort_stable(cuda_device, index_bytes):
    rng = np.random.default_rng(1)
    n, f = 9000, 9
    x = rng.integers(-3, 4, size=(n, f)).astype(np.float32)
    x[rng.random((n, f)) < 0.1] = -0.0
    x[:, 4] = rng.normal(size=n).astype(np.float32) * 1e30
    # columns of at most two distinct values take the one-pass partition:
    # one-hot, constant, {-0.0, +0.0, 3} (two keys once -0.0 folds onto +0.0), {-1, 1}
    x[:, 5] = (rng.random(n) < 0.3).astype(np.float32)
    x[:, 6] = 2.5
    x[:, 7] = rng.choice(np.array([-0.0, 0.0, 3.0], np.float32), size=n)
    x[:, 8] = rng.choice(np.array([-1.0, 1.0], np.float32), size=n)
    gp = G.GpuProblem(x, np.zeros(n, np.int64), 1, 1, index_bytes=index_bytes)
    np.testing.assert_array_equal(gp.presort_np(), O.presort(gp.x_fm_np))


@pytest.mark.parametrize("bootstrap", [False, True])
def test_bootstrap_compact(cuda_device, bootstrap):
    n, f = 5000, 6
    x, y = _data(n, f, 3, 2)
    gp = G.GpuProblem(x, y, 3, 2, bootstrap=bootstrap, seed=77)
    gl = G.GpuLists(gp, slots=2)
    ws = C.c_size_t()
    _lib.call("ct_bootstrap_workspace_size", C.byref(gp.prob), C.byref(ws))
    work = G.dev_bytes(ws.value)
    n_in = G.dev_bytes(8)
    for slot, tree in ((0, 3), (1, 11)):
        _lib.call("ct_bootstrap_compact", C.byref(gp.prob), C.byref(gl.lists), slot, tree, n_in.data_ptr(),
                  work.data_ptr(), ws.value, G.stream())
    got_n = G.from_dev(n_in, np.uint32)
    pre = gp.presort_np()
    for slot, tree in ((0, 3), (1, 11)):
        rows = O.bootstrap_rows(77, tree, n, bootstrap)
        assert int(got_n[slot]) == rows.shape[0]
        keep = np.zeros(n, bool)
        keep[rows] = True
        lists = gl.get(0, slot)
        for j in range(f):
            np.testing.assert_array_equal(lists[j, :rows.shape[0]], pre[j][keep[pre[j]]])


def _grouped_case(n, f, c, m, group_sizes, seed, integer=True, const_features=()):
    x, y = _data(n, f, c, seed, integer)
    for j in const_features:
        x[:, j] = 3.0
    rng = np.random.default_rng(seed + 100)
    perm = rng.permutation(n)
    groups, pos = [], 0
    for s in group_sizes:
        groups.append(np.sort(perm[pos:pos + s]))
        pos += s
    gp = G.GpuProblem(x, y, c, m)
    gl = G.GpuLists(gp)
    lists, starts = G.grouped_lists(gp.x_fm_np, groups)
    gl.put(0, lists)
    keys = [O.mix64(0x1234 + i) for i in range(len(groups))]
    nodes = G.node_array([dict(slot=0, start=s, n=g.shape[0], raw_id=i, key=keys[i], impurity=1.0, buf=0)
                          for i, (s, g) in enumerate(zip(starts, groups))])
    totals = np.stack([np.bincount(y[g], minlength=c) for g in groups]).astype(np.uint32)
    return gp, gl, groups, nodes, totals, keys, lists


CASES = [
    # n, f, c, m, group sizes, seed, integer-valued, constant features
    (3000, 10, 4, 3, [3000], 1, True, ()),
    (10000, 7, 7, 7, [5000, 2049, 2048, 1, 2, 3, 897], 2, True, (2,)),
    (6000, 12, 50, 5, [4100, 33, 32, 31, 1000, 804], 3, False, ()),
    (2500, 40, 2, 6, [700, 600, 500, 400, 300] , 4, True, (0, 1, 5)),
    (4000, 5, 100, 2, [4000], 5, False, ()),
]


@pytest.mark.parametrize("case", CASES)
def test_split_nodes_match_oracle(cuda_device, case):
    n, f, c, m, sizes, seed, integer, consts = case
    gp, gl, groups, nodes, totals, keys, _ = _grouped_case(n, f, c, m, sizes, seed, integer, consts)
    res, sel, _ = G.split_nodes(gp, gl, nodes, totals)
    for i, g in enumerate(groups):
        best = O.select_and_split(gp.x_fm_np, gp.y, g, totals[i].astype(np.int64), keys[i], m)
        if best is None:
            assert res[i]["feature"] == 0xFFFFFFFF, f"node {i}: GPU split where oracle has none"
            assert np.isinf(res[i]["score"])
            continue
        assert res[i]["feature"] == best.feature, f"node {i}"
        assert res[i]["pos"] == best.pos, f"node {i}"
        assert res[i]["score"] == best.score, f"node {i}"
        assert np.float32(res[i]["imp_left"]) == best.imp_left
        assert np.float32(res[i]["imp_right"]) == best.imp_right
        order, xs = O.node_sorted(gp.x_fm_np, best.feature, g)
        thr = np.float32((np.float64(xs[best.pos]) + np.float64(xs[best.pos + 1])) / 2.0)
        assert np.float32(res[i]["threshold"]) == thr


HUGE_CASES = [
    # nodes of at least 16,384 rows take k_part_seg (mark bits staged in shared
    # memory, four chains per CTA); 3,616 and 10,000 rows take k_part_big
    (50000, 6, 5, 3, [30000, 16384, 3616], 6, False, (2,)),
    (80000, 5, 3, 2, [70000, 10000], 7, True, ()),
]


@pytest.mark.parametrize("case", CASES[:4] + HUGE_CASES)
def test_partition_matches_oracle(cuda_device, case):
    n, f, c, m, sizes, seed, integer, consts = case
    gp, gl, groups, nodes, totals, keys, lists = _grouped_case(n, f, c, m, sizes, seed, integer, consts)
    res, _, res_dev = G.split_nodes(gp, gl, nodes, totals)
    G.partition_nodes(gp, gl, nodes, res_dev)
    out = gl.get(1)
    for i, g in enumerate(groups):
        if res[i]["feature"] == 0xFFFFFFFF:
            continue
        s, k = int(nodes[i]["start"]), g.shape[0]
        fstar, pos = int(res[i]["feature"]), int(res[i]["pos"])
        left = np.zeros(gp.n, bool)
        left[lists[fstar, s:s + pos + 1]] = True
        for j in range(f):
            seg = lists[j, s:s + k]
            expect = np.concatenate([seg[left[seg]], seg[~left[seg]]])
            np.testing.assert_array_equal(out[j, s:s + k], expect, err_msg=f"node {i} feature {j}")
