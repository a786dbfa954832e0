"""Parity at the benchmarked configurations, node for node against the oracle.

The small-case tests pin every kernel; these fit the workloads the bench
times, at their full sizes, and compare each tree (children, feature,
threshold, leaf class) and the forest's votes with the oracle's:

* covtype-shaped 581,012 x 54, 7 classes, max_features 7, bootstrap, uint32
  list entries carrying 20 row bits + 3 label bits: 3 trees, batched and
  plain forms, also against the committed digests;
* wide 10,000 x 3,000, 100 classes, max_features 55, uint16 entries: 2
  trees with the autotuner's options and with the extreme scan-piece and
  subtree-cutoff candidates, and the plain form;
* digits-shaped 1,797 x 64, all 50 trees, no bootstrap, max_features 8,
  bfs_threshold 4196, both forms;
* a sample of the 256-job forest queue (tiny to 34,711 rows, 2 to 48
  classes, up to 509 features), 10 trees each, through fit_forests.

The oracle trees grow in spawn-started worker processes (tests/oracle_jobs.py)
while the GPU fits run.  Reference of the split rule: dfs_module.cu:310-443,
random_tree.py:580-676; the reference's own covtype test is test_covtype.py:5-16.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from cudatree_b200 import RandomForestClassifier, synthetic
from cudatree_b200.serving import fit_forests
from oracle import cudatree_oracle as O

from . import oracle_jobs

pytestmark = pytest.mark.gpu

QUEUE_SAMPLE = (122, 152, 163, 91, 170, 2)


@pytest.fixture(scope="module")
def pool():
    with oracle_jobs.pool() as ex:
        yield ex


def _assert_same_trees(gpu_trees, oracle_trees, what):
    assert len(gpu_trees) == len(oracle_trees), what
    for i, (a, b) in enumerate(zip(gpu_trees, oracle_trees)):
        assert a.n_nodes == b.n_nodes, f"{what} tree {i}: {a.n_nodes} vs {b.n_nodes} nodes"
        np.testing.assert_array_equal(a.left_children, b.left, err_msg=f"{what} tree {i} left")
        np.testing.assert_array_equal(a.right_children, b.right, err_msg=f"{what} tree {i} right")
        np.testing.assert_array_equal(a.feature_idx_array, b.feature, err_msg=f"{what} tree {i} feature")
        np.testing.assert_array_equal(a.feature_threshold_array, b.threshold, err_msg=f"{what} tree {i} threshold")
        np.testing.assert_array_equal(a.values_array.astype(np.int64), b.value, err_msg=f"{what} tree {i} value")


def _oracle_forest(trees, classes, n_features):
    return O.Forest(trees=trees, classes=np.asarray(classes), n_features=n_features)


def test_covtype_full_size_matches_oracle(cuda_device, pool):
    fx = json.loads((Path(__file__).resolve().parent / "golden" / "covtype_trees.json").read_text())
    futs = oracle_jobs.submit_forest(pool, fx["make"], None, fx["trees"], fx["seed"], fx["max_features"],
                                     fx["bootstrap"])
    x, y = synthetic.covtype_like()
    fits = {}
    for mode in ("batched", "plain"):
        f = RandomForestClassifier(n_estimators=fx["trees"], max_features=fx["max_features"],
                                   bootstrap=fx["bootstrap"], seed=fx["seed"], fit_mode=mode).fit(x, y)
        assert f.index_bytes == 4
        fits[mode] = f
    for d, t in zip(fx["digests"], fits["batched"]._trees):
        assert t.n_nodes == d["n_nodes"]
        assert oracle_jobs.tree_digest(t.left_children, t.right_children, t.feature_idx_array,
                                       t.feature_threshold_array, t.values_array) == d["sha256"]
    ref = [fu.result() for fu in futs]
    for mode, f in fits.items():
        _assert_same_trees(f._trees, ref, f"covtype {mode}")
    xs = x[::29]
    votes = O.vote_counts(_oracle_forest(ref, fits["batched"].compt_table, 54), xs)
    np.testing.assert_array_equal(fits["batched"]._votes(xs), votes)
    np.testing.assert_array_equal(fits["batched"].predict(xs), fits["batched"].compt_table[np.argmax(votes, 1)])


def test_wide_matches_oracle_with_tuned_and_extreme_options(cuda_device, pool):
    futs = oracle_jobs.submit_forest(pool, "wide", None, 2, 12, 55, True)
    x, y = synthetic.wide()
    fits = {}
    tuned = RandomForestClassifier(n_estimators=2, max_features=55, seed=12, autotune=True).fit(x, y)
    assert tuned.index_bytes == 2 and tuned._tuned is not None
    fits[f"tuned {tuned._tuned}"] = tuned
    for piece, cut in ((4096, 128), (1024, 0)):
        f = RandomForestClassifier(n_estimators=2, max_features=55, seed=12)
        f._tuned = {"scan_piece": piece, "subtree_cutoff": cut}
        fits[f"scan_piece {piece} cutoff {cut}"] = f.fit(x, y)
    fits["plain"] = RandomForestClassifier(n_estimators=2, max_features=55, seed=12, fit_mode="plain").fit(x, y)
    ref = [fu.result() for fu in futs]
    for what, f in fits.items():
        _assert_same_trees(f._trees, ref, f"wide {what}")
    xs = x[::5]
    np.testing.assert_array_equal(tuned._votes(xs), O.vote_counts(_oracle_forest(ref, tuned.compt_table, 3000), xs))


def test_digits_shaped_all_50_trees_match_oracle(cuda_device, pool):
    futs = oracle_jobs.submit_forest(pool, "digits_like", None, 50, 11, 8, False)
    x, y = synthetic.digits_like()
    fits = {mode: RandomForestClassifier(n_estimators=50, max_features=8, bootstrap=False, seed=11,
                                         fit_mode=mode).fit(x, y, bfs_threshold=4196)
            for mode in ("batched", "plain")}
    ref = [fu.result() for fu in futs]
    for mode, f in fits.items():
        _assert_same_trees(f._trees, ref, f"digits {mode}")
        assert int((f.predict(x) != y).sum()) == 0  # memorize (test_digits.py:10-17)
    np.testing.assert_array_equal(fits["batched"]._votes(x),
                                  O.vote_counts(_oracle_forest(ref, fits["batched"].compt_table, 64), x))


def test_forest_queue_sample_matches_oracle(cuda_device, pool):
    futs = {j: oracle_jobs.submit_forest(pool, "blob_job", j, 10, j, None, True) for j in QUEUE_SAMPLE}
    jobs = [synthetic.blob_job(j) for j in QUEUE_SAMPLE]
    forests = fit_forests(jobs, n_estimators=10, seeds=QUEUE_SAMPLE)
    for j, (x, y), f in zip(QUEUE_SAMPLE, jobs, forests):
        ref = [fu.result() for fu in futs[j]]
        _assert_same_trees(f._trees, ref, f"queue job {j} {x.shape}")
        xs = x[: min(4000, x.shape[0])]
        np.testing.assert_array_equal(f.predict(xs), O.predict(_oracle_forest(ref, np.unique(y), x.shape[1]), xs))
