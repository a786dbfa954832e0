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
