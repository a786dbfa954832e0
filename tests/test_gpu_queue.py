"""Forest queue through shared level steps (ct_fit_queue): every job's trees
are the ones its solo fit grows and the oracle's, whatever mix of sizes,
feature counts, class counts and index widths shares the launches (the
reference fits such a queue job by job, hybridforest/builder.py:79-141)."""
import numpy as np
import pytest

from cudatree_b200 import RandomForestClassifier
from cudatree_b200.forest_queue import fit_forests
from oracle import cudatree_oracle as O

pytestmark = pytest.mark.gpu


def _blobs(n, f, c, seed, ties=False):
    rng = np.random.default_rng(seed)
    y = rng.integers(0, c, size=n)
    means = rng.normal(scale=1.5, size=(c, f))
    x = (rng.normal(size=(n, f)) + means[y]).astype(np.float32)
    if ties:
        x[:, ::2] = np.round(x[:, ::2])
    return x, y


def _same(a, b):
    assert len(a._trees) == len(b._trees)
    for s, t in zip(a._trees, b._trees):
        np.testing.assert_array_equal(s.left_children, t.left_children)
        np.testing.assert_array_equal(s.feature_idx_array, t.feature_idx_array)
        np.testing.assert_array_equal(s.feature_threshold_array, t.feature_threshold_array)
        np.testing.assert_array_equal(s.values_array.astype(np.int64), t.values_array.astype(np.int64))


def test_mixed_queue_matches_solo_fits_and_oracle(cuda_device):
    """Jobs of 20 to 70,000 rows (16- and 32-bit lists: two groups), 3 to 130
    features (constant-feature masks on for groups of at most 64 features),
    one to 40 classes, and a job all of whose nodes go to warp subtrees."""
    specs = [(20, 5, 1), (900, 70, 5), (3000, 30, 3), (70000, 6, 4), (40, 3, 2), (5000, 130, 40), (1500, 12, 7)]
    jobs = [_blobs(n, f, c, 300 + k, ties=k % 2 == 0) for k, (n, f, c) in enumerate(specs)]
    seeds = [500 + k for k in range(len(jobs))]
    got = fit_forests(jobs, n_estimators=4, seeds=seeds)
    for (x, y), seed, g in zip(jobs, seeds, got):
        solo = RandomForestClassifier(n_estimators=4, seed=seed).fit(x, y)
        _same(g, solo)
        np.testing.assert_array_equal(g.predict(x[:2000]), solo.predict(x[:2000]))
    for k in (0, 2, 4, 6):
        x, y = jobs[k]
        ref = O.fit_forest(x, y, n_estimators=4, seed=seeds[k])
        for t, r in zip(got[k]._trees, ref.trees):
            np.testing.assert_array_equal(t.left_children, r.left)
            np.testing.assert_array_equal(t.feature_idx_array, r.feature)
            np.testing.assert_array_equal(t.feature_threshold_array, r.threshold)


def test_queue_groups_within_a_memory_budget(cuda_device):
    """A small group budget splits the queue into several shared fits; the
    trees do not change."""
    jobs = [_blobs(600 + 97 * k, 9 + k, 3 + k % 4, 40 + k) for k in range(6)]
    a = fit_forests(jobs, n_estimators=3, seeds=range(6))
    b = fit_forests(jobs, n_estimators=3, seeds=range(6), group_bytes=1)
    for fa, fb in zip(a, b):
        _same(fa, fb)
