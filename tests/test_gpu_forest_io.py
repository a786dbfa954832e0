"""Forest input checks on the device path: ct_predict / ct_predict_compact
check a caller's forest before walking it, and the server checks forests it
is given; a malformed forest gets CT_ERR_ARG, and the next call with a good
forest still predicts as the oracle does."""
import ctypes as C

import numpy as np
import pytest
import torch

from cudatree_b200 import CudaTreeError, RandomForestClassifier, _lib
from cudatree_b200.random_forest import PACKED_DTYPE, pack_trees
from cudatree_b200.serving import ForestServer
from oracle import cudatree_oracle as O

pytestmark = pytest.mark.gpu


def _data(n=3000, f=6, c=4, seed=3):
    rng = np.random.default_rng(seed)
    y = rng.integers(0, c, size=n)
    x = (rng.normal(size=(n, f)) + rng.normal(scale=1.5, size=(c, f))[y]).astype(np.float32)
    return x, y


def _predict_dev(packed, offsets, x, n_features, n_classes, compact):
    dev = torch.device("cuda", 0)
    nodes = torch.from_numpy(np.ascontiguousarray(packed).view(np.uint8).copy()).to(dev)
    offs = torch.from_numpy(np.ascontiguousarray(offsets, np.uint32)).to(dev)
    xd = torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(dev)
    pred = torch.empty(x.shape[0], dtype=torch.int32, device=dev)
    votes = torch.empty((x.shape[0], n_classes), dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    lib = _lib.load()
    n_nodes = packed.shape[0]
    if compact:
        out = torch.empty(n_nodes * 8, dtype=torch.uint8, device=dev)
        rc = lib.ct_compact_forest(nodes.data_ptr(), n_nodes, n_features, n_nodes, out.data_ptr(), st)
        assert rc == 0, _lib.last_error()
        rc = lib.ct_predict_compact(out.data_ptr(), n_nodes, offs.data_ptr(), offsets.shape[0], xd.data_ptr(),
                                    x.shape[0], n_features, n_classes, votes.data_ptr(), pred.data_ptr(), st)
    else:
        rc = lib.ct_predict(nodes.data_ptr(), n_nodes, offs.data_ptr(), offsets.shape[0], xd.data_ptr(), x.shape[0],
                            n_features, n_classes, votes.data_ptr(), pred.data_ptr(), st)
    torch.cuda.synchronize()
    return rc, pred.cpu().numpy()


def _malformed(packed, offsets, case):
    p, off = packed.copy(), offsets.copy()
    inner = np.flatnonzero(p["left"][off[1]:] != 0) + off[1]  # inner nodes of tree 1
    leaf = int(np.flatnonzero(p["left"][off[1]:] == 0)[0] + off[1])
    if case == "cycle":
        deep = int(inner[-1])
        p["left"][deep] = 1  # points back towards its tree's root
    elif case == "child_past_tree":
        root = int(off[1])
        p["left"][root] = off[2] - off[1] - 1  # right child = first node of the next tree
    elif case == "bad_feature":
        p["feature"][int(inner[0])] = 999
    elif case == "bad_class":
        p["value"][leaf] = 77
    elif case == "offsets_out_of_order":
        off[1], off[2] = off[2], off[1]
    return p, off


@pytest.mark.parametrize("compact", [False, True])
@pytest.mark.parametrize("case", ["cycle", "child_past_tree", "bad_feature", "bad_class", "offsets_out_of_order"])
def test_predict_refuses_malformed_forests(cuda_device, case, compact):
    x, y = _data()
    forest = RandomForestClassifier(n_estimators=4, seed=9).fit(x, y)
    packed, offsets = pack_trees(forest._trees)
    bad, bad_off = _malformed(packed, offsets, case)
    rc, _ = _predict_dev(bad, bad_off, x[:100], 6, forest.n_labels, compact)
    assert rc == 1, case
    assert "malformed forest" in _lib.last_error()
    rc, pred = _predict_dev(packed, offsets, x[:500], 6, forest.n_labels, compact)
    assert rc == 0, _lib.last_error()
    ref = O.Forest(trees=[O.Tree(t.left_children, t.right_children, t.feature_idx_array,
                                 t.feature_threshold_array, t.values_array.astype(np.int64))
                          for t in forest._trees], classes=np.arange(forest.n_labels), n_features=6)
    np.testing.assert_array_equal(pred, O.predict(ref, x[:500]))


def test_server_refuses_malformed_forests(cuda_device):
    x, y = _data()
    forest = RandomForestClassifier(n_estimators=4, seed=9).fit(x, y)
    packed, offsets = pack_trees(forest._trees)
    srv = ForestServer(max_features=16, fit_workers=1, max_fit_rows=1000, max_fit_trees=2)
    try:
        for case in ("cycle", "child_past_tree", "bad_feature", "bad_class", "offsets_out_of_order"):
            bad, bad_off = _malformed(packed, offsets, case)
            with pytest.raises(CudaTreeError, match="malformed forest"):
                srv.add_packed(bad, bad_off, 6, forest.n_labels)
        fid = srv.add_forest(forest)
        np.testing.assert_array_equal(srv.predict(fid, x[:300]), forest.predict(x[:300]))
    finally:
        srv.close()


def test_stored_forest_predicts_as_fitted(cuda_device, tmp_path):
    """fit -> pickle / flat bytes / file -> restore -> predict and
    predict_proba equal the fitted forest's and the oracle's, vote for vote;
    the stored bytes also load straight into a server's forest pool.  The
    reference's restored forest cannot predict (random_forest.py:18-23,
    :94, :453-457)."""
    import pickle

    x, y = _data(4000, 9, 5, 21)
    labels = np.array(["oak", "elm", "ash", "fir", "yew"])[y]
    forest = RandomForestClassifier(n_estimators=7, seed=33).fit(x, labels)
    ref = O.fit_forest(x, labels, n_estimators=7, seed=33)
    want = forest.predict(x)
    np.testing.assert_array_equal(want, O.predict(ref, x))
    forest.save(tmp_path / "f.ctf")
    restored = [pickle.loads(pickle.dumps(forest)), RandomForestClassifier.from_bytes(forest.to_bytes()),
                RandomForestClassifier.load(tmp_path / "f.ctf")]
    for g in restored:
        np.testing.assert_array_equal(g.predict(x), want)
        np.testing.assert_array_equal(g.predict_proba(x), forest.predict_proba(x))
        np.testing.assert_array_equal(g.predict_proba(x), O.predict_proba(ref, x))
    srv = ForestServer(max_features=16, fit_workers=1, max_fit_rows=1000, max_fit_trees=2)
    try:
        fid = srv.load_forest(forest.to_bytes())
        np.testing.assert_array_equal(srv.predict(fid, x[:1500]), want[:1500])
        fid2 = srv.load_forest(tmp_path / "f.ctf")
        np.testing.assert_array_equal(srv.predict(fid2, x[1500:]), want[1500:])
    finally:
        srv.close()
