"""ct_split_nodes_noalloc against ct_split_nodes.

The allocation-free entry point serves callers that cannot hand the library
device memory (another allocator owns the device's memory, a latency-bound
loop must not call cudaMalloc/cudaFree, or a C FFI host owns no device
buffers).  Its scratch is a static per-device array shared by every call, so
this test runs it twice in a row on different node batches and checks each
result field for field against the workspace-based entry point (the split
search is exact: integer positions, fp64 scores, fp32 impurities compared
with ==).  This file is collected last so that a failure here does not stop
a `-x` run before the other tests have run.
"""
import ctypes as C

import numpy as np
import pytest

from cudatree_b200 import _lib

from . import gpu_utils as G
from .test_gpu_kernels import _grouped_case

pytestmark = pytest.mark.gpu

BATCHES = [
    (10000, 7, 7, 7, [5000, 2049, 2048, 1, 2, 3, 897], 2, True, (2,)),
    (6000, 12, 50, 5, [4100, 33, 32, 31, 1000, 804], 3, False, ()),
]


def _noalloc(gp, gl, nodes, totals):
    nn = nodes.shape[0]
    nd = G.to_dev(nodes)
    td = G.to_dev(totals.astype(np.uint32))
    out = G.dev_bytes(nn * 32)
    _lib.call("ct_split_nodes_noalloc", C.byref(gp.prob), C.byref(gl.lists), nd.data_ptr(), td.data_ptr(), nn,
              int(nodes["n"].sum()), out.data_ptr(), G.stream())
    return G.from_dev(out[:nn * 32], np.dtype(_lib.SPLIT_DTYPE_FIELDS))


def test_noalloc_matches_workspace_split_twice_in_a_row(cuda_device):
    for case in BATCHES:
        gp, gl, groups, nodes, totals, keys, _ = _grouped_case(*case)
        ref, _, _ = G.split_nodes(gp, gl, nodes, totals)
        got = _noalloc(gp, gl, nodes, totals)
        for field in ("score", "feature", "pos", "imp_left", "imp_right", "threshold", "n_selected"):
            np.testing.assert_array_equal(got[field], ref[field], err_msg=field)


def test_noalloc_rejects_batches_beyond_the_static_scratch(cuda_device):
    gp, gl, groups, nodes, totals, keys, _ = _grouped_case(*BATCHES[0])
    nd = G.to_dev(nodes)
    td = G.to_dev(totals.astype(np.uint32))
    out = G.dev_bytes(nodes.shape[0] * 32)
    st = _lib.load().ct_split_nodes_noalloc(C.byref(gp.prob), C.byref(gl.lists), nd.data_ptr(), td.data_ptr(),
                                            nodes.shape[0], 1 << 34, out.data_ptr(), G.stream())
    assert st == 1
    assert "static scratch" in _lib.last_error()


def test_noalloc_understated_total_samples_then_recovers(cuda_device):
    """total_samples sizes every scratch list.  Passed 1 for a batch of 10,000
    rows, the device capacity checks stop the split search (no record past a
    list's end is written or read) and the call returns CT_ERR_CAPACITY; the
    next call with the right total, which reuses the same static scratch,
    matches ct_split_nodes field for field."""
    gp, gl, groups, nodes, totals, keys, _ = _grouped_case(*BATCHES[0])
    nd = G.to_dev(nodes)
    td = G.to_dev(totals.astype(np.uint32))
    out = G.dev_bytes(nodes.shape[0] * 32)
    st = _lib.load().ct_split_nodes_noalloc(C.byref(gp.prob), C.byref(gl.lists), nd.data_ptr(), td.data_ptr(),
                                            nodes.shape[0], 1, out.data_ptr(), G.stream())
    assert st == 7
    assert "work lists overflowed" in _lib.last_error()
    ref, _, _ = G.split_nodes(gp, gl, nodes, totals)
    got = _noalloc(gp, gl, nodes, totals)
    for field in ("score", "feature", "pos", "imp_left", "imp_right", "threshold", "n_selected"):
        np.testing.assert_array_equal(got[field], ref[field], err_msg=field)
