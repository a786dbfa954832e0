"""cudatree_b200: B200-native random-forest fit + predict behind CudaTree's API.

``from cudatree_b200 import RandomForestClassifier`` gives the reference's
``RandomForestClassifier(n_estimators, max_features, min_samples_split,
bootstrap).fit(x, y, bfs_threshold).predict(x)`` surface
(EasonLiao/CudaTree ``cudatree/__init__.py``).
"""
from ._lib import CudaTreeError, version
from .random_forest import RandomForestClassifier, restore_forest
from .random_tree import RandomClassifierTree, restore_tree

__version__ = "0.1.0"

__all__ = ["RandomForestClassifier", "RandomClassifierTree", "restore_forest", "restore_tree",
           "CudaTreeError", "version", "__version__"]
