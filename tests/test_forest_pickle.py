"""Pickling of a fitted forest (reference random_forest.py:18-23 and
random_tree.py:21-36): the trees, the label table and the constructor
arguments survive a round trip, and the trees belong to the restored forest.
Built from node arrays on the host, so no GPU is needed."""
import pickle

import numpy as np

from cudatree_b200 import RandomForestClassifier


def _forest():
    f = RandomForestClassifier(n_estimators=2, max_features=3, bootstrap=False, seed=7)
    f.dtype_labels = np.dtype(np.uint8)
    f.n_features = 4
    f.compt_table = np.array([3, 5, 9])
    f.n_labels = 3
    trees = []
    for k in range(2):
        trees.append(f._make_tree(np.array([1, 0, 0], np.uint32), np.array([2, 0, 0], np.uint32),
                                  np.array([2 + k, 0, 0], np.uint16), np.array([0.5 * (k + 1), 0, 0], np.float32),
                                  np.array([0, 1, 2], np.uint32)))
    f._trees = trees
    return f


def test_pickle_round_trip_keeps_trees_labels_and_arguments():
    f = _forest()
    g = pickle.loads(pickle.dumps(f))
    assert isinstance(g, RandomForestClassifier)
    assert (g.n_estimators, g.max_features, g.bootstrap, g.seed, g.n_features) == (2, 3, False, 7, 4)
    np.testing.assert_array_equal(g.compt_table, f.compt_table)
    assert g.n_labels == 3 and g.dtype_labels == np.uint8
    assert len(g._trees) == 2
    for a, b in zip(f._trees, g._trees):
        for name in ("left_children", "right_children", "feature_idx_array", "feature_threshold_array",
                     "values_array"):
            np.testing.assert_array_equal(getattr(a, name), getattr(b, name))
        assert b.values_array.dtype == np.uint8
        assert b.forest is g


def test_flat_format_round_trip_and_pickle_use_it():
    """to_bytes/from_bytes and pickling write the versioned flat format: the
    node section is the ct_packed_node array, the label table and the
    constructor arguments come back, and the trees belong to the new forest."""
    import struct

    from cudatree_b200 import forest_format
    f = _forest()
    data = f.to_bytes()
    assert data[:8] == b"CTFOREST" and struct.unpack_from("<I", data, 8)[0] == forest_format.VERSION
    for g in (RandomForestClassifier.from_bytes(data), pickle.loads(pickle.dumps(f))):
        assert (g.n_estimators, g.max_features, g.bootstrap, g.seed, g.n_features) == (2, 3, False, 7, 4)
        np.testing.assert_array_equal(g.compt_table, f.compt_table)
        for a, b in zip(f._trees, g._trees):
            for name in ("left_children", "right_children", "feature_idx_array", "feature_threshold_array",
                         "values_array"):
                np.testing.assert_array_equal(getattr(a, name), getattr(b, name))
            assert b.forest is g
    assert pickle.dumps(f).count(b"CTFOREST") == 1


def test_flat_format_string_labels_and_files(tmp_path):
    f = _forest()
    f.compt_table = np.array(["ash", "birch", "cedar"])
    f.save(tmp_path / "forest.ctf")
    g = RandomForestClassifier.load(tmp_path / "forest.ctf")
    np.testing.assert_array_equal(g.compt_table, f.compt_table)


def test_flat_format_rejects_corrupt_and_malformed_data():
    import struct
    import zlib

    import pytest

    from cudatree_b200 import forest_format
    f = _forest()
    data = bytearray(f.to_bytes())
    bad = bytearray(data)
    bad[40] ^= 1
    with pytest.raises(ValueError, match="CRC|header"):
        forest_format.loads(bytes(bad))
    with pytest.raises(ValueError, match="magic"):
        forest_format.loads(b"NOTATREE" + bytes(data[8:]))
    v2 = bytearray(data)
    struct.pack_into("<I", v2, 8, 2)
    with pytest.raises(ValueError, match="version 2"):
        forest_format.loads(bytes(v2))
    # a node pointing at itself, stored with a valid CRC: the node check refuses it
    packed, offsets = np.zeros(3, forest_format.PACKED_DTYPE), np.array([0], np.uint32)
    packed["left"] = [1, 0, 0]
    good = forest_format.encode(packed, offsets, 4, 3, np.arange(3), {})
    forest_format.loads(good)  # a stump: valid
    packed["left"][1] = 1
    cyc = forest_format.encode(packed, offsets, 4, 3, np.arange(3), {})
    assert struct.unpack_from("<I", cyc, len(cyc) - 4)[0] == zlib.crc32(cyc[:-4]) & 0xFFFFFFFF
    with pytest.raises(ValueError, match="malformed forest"):
        forest_format.loads(cyc)
    with pytest.raises(ValueError, match="not fitted"):
        RandomForestClassifier(3).to_bytes()


def test_unfitted_forest_pickles_as_its_arguments():
    f = RandomForestClassifier(n_estimators=5, max_features=2, seed=4)
    g = pickle.loads(pickle.dumps(f))
    assert (g.n_estimators, g.max_features, g.seed, g._trees) == (5, 2, 4, [])
