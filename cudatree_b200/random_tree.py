"""One fitted tree in the reference's node-array format.

Mirrors ``cudatree/random_tree.py`` / ``cudatree/base_tree.py``: the arrays
``left_children`` / ``right_children`` (uint32, 0 = leaf),
``feature_idx_array`` (uint16), ``feature_threshold_array`` (float32) and
``values_array`` (label dtype) of ``random_tree.py:284-289``, root at 0.
Unlike the reference, nodes are numbered breadth-first (left child before
right child), so the right child of node i is always ``left_children[i] + 1``.
"""
from __future__ import annotations

import numpy as np


def restore_tree(left_children, right_children, feature_threshold_array, values_array,
                 feature_idx_array, dtype_labels, n_features):
    """Unpickle hook (reference random_tree.py:21-36)."""
    tree = RandomClassifierTree()
    tree.left_children = left_children
    tree.right_children = right_children
    tree.feature_threshold_array = feature_threshold_array
    tree.values_array = values_array
    tree.feature_idx_array = feature_idx_array
    tree.dtype_labels = np.dtype(dtype_labels)
    tree.n_features = n_features
    return tree


class RandomClassifierTree:
    """A fitted classification tree (node arrays in breadth-first order)."""

    def __init__(self, forest=None):
        self.left_children = None
        self.right_children = None
        self.feature_idx_array = None
        self.feature_threshold_array = None
        self.values_array = None
        self.dtype_labels = np.dtype(np.uint8)
        self.forest = forest
        self.n_features = getattr(forest, "n_features", None) if forest is not None else None

    def fit(self, samples, target, sorted_indices, n_samples):
        """Grow one tree of a forest prepared by fit_init, the per-tree call
        hybridforest's GPU worker makes (hybridforest/builder.py:129-132,
        random_tree.py:461-491).  sorted_indices is what the forest's
        _get_sorted_indices returned (the tree's index: its bootstrap sample is
        drawn inside the fit from the forest's seed); samples, target and
        n_samples are accepted for the reference's signature."""
        f = self.forest
        if f is None or getattr(f, "_x_fm", None) is None:
            raise ValueError("the forest has no data: call forest.fit_init(samples, target) first")
        grown = f._fit_trees(int(sorted_indices), 1, f.fit_mode, f.bfs_threshold)[0]
        for name in ("left_children", "right_children", "feature_idx_array", "feature_threshold_array",
                     "values_array", "dtype_labels", "n_features"):
            setattr(self, name, getattr(grown, name))
        return self

    @property
    def n_nodes(self) -> int:
        return 0 if self.left_children is None else int(self.left_children.shape[0])

    def __reduce__(self):
        assert self.left_children is not None, "tree is not fitted"
        return restore_tree, (self.left_children, self.right_children, self.feature_threshold_array,
                              self.values_array, self.feature_idx_array, self.dtype_labels.str,
                              self.n_features)

    def print_tree(self):
        """Indented dump of the tree (reference base_tree.py:13-25)."""
        def rec(i, depth):
            if self.left_children[i] == 0 and self.right_children[i] == 0:
                print("[LEAF] Depth: %s, Value: %s" % (depth, self.values_array[i]))
            else:
                print("[NODE] Depth: %s, Feature: %s, Threshold: %f" %
                      (depth, self.feature_idx_array[i], self.feature_threshold_array[i]))
                rec(int(self.left_children[i]), depth + 1)
                rec(int(self.right_children[i]), depth + 1)
        rec(0, 0)

    def depth(self) -> int:
        d = np.zeros(self.n_nodes, dtype=np.int64)
        inner = np.nonzero(self.left_children)[0]
        for i in inner:  # breadth-first order: parents precede children
            d[self.left_children[i]] = d[i] + 1
            d[self.right_children[i]] = d[i] + 1
        return int(d.max()) if d.size else 0

    def gpu_predict(self, inputs):
        """Class ids predicted by this tree alone (reference base_tree.py:44-81)."""
        from .random_forest import _predict_packed, pack_trees
        packed, offsets = pack_trees([self])
        votes = _predict_packed(packed, offsets, 1, inputs, self.n_features,
                                int(self.values_array.max()) + 1 if self.n_nodes else 1,
                                want_votes=False)
        return votes.astype(self.dtype_labels)
