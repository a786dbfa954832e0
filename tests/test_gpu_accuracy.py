"""Accuracy against scikit-learn, the reference's statistical test
(test/helpers.py:4-28, called by test_digits.py:20-21, test_iris.py:17-18 and
test_diabetes_classify.py:17-19): train 11-tree forests on the first half,
score the second half, 10 repeats, and require the summed score to be at least
0.98 of scikit-learn's.  Both forests are seeded per repeat, so the outcome is
fixed."""
import numpy as np
import pytest
from sklearn.datasets import load_diabetes, load_digits, load_iris
from sklearn.ensemble import RandomForestClassifier as SkRF

from cudatree_b200 import RandomForestClassifier

pytestmark = pytest.mark.gpu

DATASETS = {
    "digits": lambda: (load_digits().data, load_digits().target),
    "iris": lambda: (load_iris().data, load_iris().target),
    "diabetes": lambda: (load_diabetes().data, load_diabetes().target > 140),
}


@pytest.mark.parametrize("name", sorted(DATASETS))
def test_accuracy_vs_sklearn(cuda_device, name):
    x, y = DATASETS[name]()
    n = x.shape[0] // 2
    ours = theirs = 0.0
    for i in range(10):
        forest = RandomForestClassifier(n_estimators=11, bootstrap=True, seed=i).fit(x[:n], y[:n])
        ours += forest.score(x[n:], y[n:])
        theirs += SkRF(n_estimators=11, bootstrap=True, random_state=i).fit(x[:n], y[:n]).score(x[n:], y[n:])
    assert ours >= 0.98 * theirs, f"mean accuracy {ours / 10:.4f} vs scikit-learn {theirs / 10:.4f}"
