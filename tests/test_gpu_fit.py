"""Whole-forest parity: plain and batched fits against the oracle, tree for
tree and node for node, plus predict votes and the reference's memorize KATs."""
import numpy as np
import pytest
from sklearn.datasets import load_diabetes, load_digits, load_iris

from cudatree_b200 import RandomForestClassifier
from oracle import cudatree_oracle as O

pytestmark = pytest.mark.gpu


def _assert_same_trees(gpu_trees, oracle_trees):
    assert len(gpu_trees) == len(oracle_trees)
    for i, (a, b) in enumerate(zip(gpu_trees, oracle_trees)):
        assert a.n_nodes == b.n_nodes, f"tree {i}: {a.n_nodes} vs {b.n_nodes} nodes"
        np.testing.assert_array_equal(a.left_children, b.left, err_msg=f"tree {i} left")
        np.testing.assert_array_equal(a.right_children, b.right, err_msg=f"tree {i} right")
        np.testing.assert_array_equal(a.feature_idx_array, b.feature, err_msg=f"tree {i} feature")
        np.testing.assert_array_equal(a.feature_threshold_array, b.threshold, err_msg=f"tree {i} thr")
        np.testing.assert_array_equal(a.values_array.astype(np.int64), b.value, err_msg=f"tree {i} value")


def _synthetic(n, f, c, seed):
    rng = np.random.default_rng(seed)
    y = rng.integers(0, c, size=n)
    means = rng.normal(scale=1.5, size=(c, f))
    x = (rng.normal(size=(n, f)) + means[y]).astype(np.float32)
    x[:, ::3] = np.round(x[:, ::3])  # ties
    return x, y


DATASETS = {
    "iris": lambda: (load_iris().data, load_iris().target),
    "digits": lambda: (load_digits().data, load_digits().target),
    "synthetic7": lambda: _synthetic(3000, 9, 7, 5),
}


@pytest.mark.parametrize("mode", ["plain", "batched"])
@pytest.mark.parametrize("name,bootstrap", [("iris", False), ("digits", True), ("synthetic7", True)])
def test_fit_matches_oracle(cuda_device, name, bootstrap, mode):
    x, y = DATASETS[name]()
    forest = RandomForestClassifier(n_estimators=3, bootstrap=bootstrap, seed=123, fit_mode=mode)
    forest.fit(x, y, bfs_threshold=500)
    ref = O.fit_forest(x, y, n_estimators=3, bootstrap=bootstrap, seed=123)
    _assert_same_trees(forest._trees, ref.trees)
    np.testing.assert_array_equal(forest.predict(x), O.predict(ref, x))
    np.testing.assert_array_equal(forest.predict_proba(x), O.predict_proba(ref, x))


@pytest.mark.parametrize("mode", ["plain", "batched"])
@pytest.mark.parametrize("n,f,c", [(4096, 8, 16), (4097, 8, 16), (66000, 6, 3), (2000, 5, 1)])
def test_label_carrying_lists_match_oracle(cuda_device, n, f, c, mode):
    """The fit's lists carry each row's label above its row id when both fit
    one index entry.  4,096 rows (12 bits) and 16 classes (4 bits) fill a
    16-bit entry; 4,097 rows need 13 bits, so those lists hold plain row ids;
    66,000 rows take 32-bit entries (17 + 2 bits); one class needs no label
    bits.  Every form grows the oracle's trees."""
    x, y = _synthetic(n, f, max(c, 1), 11)
    forest = RandomForestClassifier(n_estimators=2, bootstrap=True, seed=5, fit_mode=mode)
    forest.fit(x, y, bfs_threshold=1000)
    ref = O.fit_forest(x, y, n_estimators=2, bootstrap=True, seed=5)
    _assert_same_trees(forest._trees, ref.trees)
    np.testing.assert_array_equal(forest.predict(x), O.predict(ref, x))


def test_bootstrap_of_more_than_128_trees_matches_oracle(cuda_device):
    """The bootstrap compacts at most 128 trees per pass over the presort:
    140 trees in flight take two passes, and every tree is the oracle's."""
    x, y = _synthetic(600, 5, 3, 13)
    forest = RandomForestClassifier(n_estimators=140, bootstrap=True, seed=21, fit_mode="batched")
    forest.fit(x, y)
    ref = O.fit_forest(x, y, n_estimators=140, bootstrap=True, seed=21)
    _assert_same_trees(forest._trees, ref.trees)


def test_plain_equals_batched_large(cuda_device):
    x, y = _synthetic(70000, 12, 5, 9)  # uint32 indices
    a = RandomForestClassifier(n_estimators=4, seed=7, fit_mode="plain").fit(x, y)
    b = RandomForestClassifier(n_estimators=4, seed=7, fit_mode="batched").fit(x, y)
    for ta, tb in zip(a._trees, b._trees):
        np.testing.assert_array_equal(ta.left_children, tb.left_children)
        np.testing.assert_array_equal(ta.feature_idx_array, tb.feature_idx_array)
        np.testing.assert_array_equal(ta.feature_threshold_array, tb.feature_threshold_array)
        np.testing.assert_array_equal(ta.values_array, tb.values_array)


@pytest.mark.parametrize("name", ["iris", "digits", "diabetes"])
def test_memorize(cuda_device, name):
    """Reference known-answer tests: test_iris.py:7-14, test_digits.py:10-17,
    test_diabetes_classify.py:7-14 (bootstrap=False, zero training errors)."""
    if name == "diabetes":
        x, y = load_diabetes().data, load_diabetes().target > 140
    else:
        x, y = DATASETS[name]()
    forest = RandomForestClassifier(n_estimators=6, bootstrap=False, seed=3)
    forest.fit(x, y)
    assert int((forest.predict(x) != y).sum()) == 0


@pytest.mark.parametrize("mode", ["plain", "batched"])
def test_golden_forests(cuda_device, mode):
    """Committed canonical forests (tests/golden/oracle_forests.npz) node for node."""
    from pathlib import Path
    from tests.golden.make_golden import FOREST_CASES
    g = np.load(Path(__file__).resolve().parent / "golden" / "oracle_forests.npz")
    for name, (make, t, bs, m, seed) in FOREST_CASES.items():
        x, y = make()
        forest = RandomForestClassifier(n_estimators=t, bootstrap=bs, max_features=m, seed=seed, fit_mode=mode)
        forest.fit(x, y)
        for i, tr in enumerate(forest._trees):
            np.testing.assert_array_equal(tr.left_children, g[f"{name}/{i}/left"])
            np.testing.assert_array_equal(tr.right_children, g[f"{name}/{i}/right"])
            np.testing.assert_array_equal(tr.feature_idx_array, g[f"{name}/{i}/feature"])
            np.testing.assert_array_equal(tr.feature_threshold_array, g[f"{name}/{i}/threshold"])
            np.testing.assert_array_equal(tr.values_array.astype(np.int64), g[f"{name}/{i}/value"])


@pytest.mark.parametrize("n,f,c,seed", [(1797, 64, 10, 0), (3000, 3000, 7, 1), (20000, 5, 3, 2)])
def test_compact_nodes_match_packed_and_oracle(cuda_device, n, f, c, seed):
    """8-byte compact nodes give the same votes as packed nodes and the oracle
    (feature bits from 3 to 12; deep trees from noisy labels)."""
    x, y = _synthetic(n, f, c, seed)
    if seed == 2:
        y = np.random.default_rng(5).integers(0, c, size=n)  # noise labels: deep trees
    forest = RandomForestClassifier(n_estimators=12, seed=seed).fit(x, y)
    assert forest._compact_fits()
    xs = np.concatenate([x[:2000], np.random.default_rng(9).normal(size=(500, f)).astype(np.float32)])
    packed = forest._votes(xs, compact=False)
    compact = forest._votes(xs, compact=True)
    np.testing.assert_array_equal(compact, packed)
    ref = O.Forest(trees=[O.Tree(t.left_children, t.right_children, t.feature_idx_array,
                                 t.feature_threshold_array, t.values_array.astype(np.int64))
                          for t in forest._trees], classes=forest.compt_table, n_features=f)
    np.testing.assert_array_equal(compact, O.vote_counts(ref, xs))


@pytest.mark.parametrize("mss", [1, 3])
def test_warp_subtrees_grow_the_same_trees(cuda_device, mss):
    """Nodes of at most subtree_cutoff rows are grown whole by one warp (one
    row per lane up to 32, four rows per lane up to 128); the trees must equal
    those of the level steps alone (cutoff 0) and the oracle's, for deep trees
    (noise labels), ties and min_samples_split."""
    rng = np.random.default_rng(1031)  # labels independent of x
    x, _ = _synthetic(1500, 24, 5, 31)
    y = rng.integers(0, 5, size=1500)
    forests = {}
    for cut in (0, 8, 32, 64, 128):
        forests[cut] = RandomForestClassifier(n_estimators=4, min_samples_split=mss, seed=77,
                                              subtree_cutoff=cut).fit(x, y)
    for cut in (8, 32, 64, 128):
        for a, b in zip(forests[cut]._trees, forests[0]._trees):
            np.testing.assert_array_equal(a.left_children, b.left_children)
            np.testing.assert_array_equal(a.feature_idx_array, b.feature_idx_array)
            np.testing.assert_array_equal(a.feature_threshold_array, b.feature_threshold_array)
            np.testing.assert_array_equal(a.values_array, b.values_array)
    ref = O.fit_forest(x, y, n_estimators=4, min_samples_split=mss, seed=77)
    _assert_same_trees(forests[32]._trees, ref.trees)
    _assert_same_trees(forests[128]._trees, ref.trees)


def test_nan_samples_are_rejected(cuda_device):
    """The device transpose flags NaN; the fit raises and a clean fit still works."""
    x, y = _synthetic(500, 6, 3, 5)
    bad = x.copy()
    bad[123, 4] = np.nan
    with pytest.raises(ValueError, match="NaN"):
        RandomForestClassifier(n_estimators=2, seed=1).fit(bad, y)
    ok = RandomForestClassifier(n_estimators=2, seed=1).fit(x, y)
    ref = O.fit_forest(x, y, n_estimators=2, seed=1)
    _assert_same_trees(ok._trees, ref.trees)


def test_autotune_keeps_the_trees(cuda_device):
    """The autotuner only picks among options that grow the same trees."""
    x, y = _synthetic(4000, 12, 4, 9)
    tuned = RandomForestClassifier(n_estimators=6, seed=5, autotune=True).fit(x, y)
    assert tuned._tuned is not None and tuned._tuned["scan_piece"] in (1024, 2048, 4096)
    assert tuned._tuned["subtree_cutoff"] in (0, 32, 128)
    assert tuned._tuned["part_shape"] in range(4) and tuned._tuned["huge_rows"] in (0, 16384, 0xFFFFFFFF)
    assert tuned._tuned["small_rows"] in (0, 512, 2048, 8192)
    # a later forest of the same shape takes the stored choice (the tune cache)
    again = RandomForestClassifier(n_estimators=6, seed=5, autotune=True).fit(x, y)
    assert again._tuned == tuned._tuned
    ref = RandomForestClassifier(n_estimators=6, seed=5).fit(x, y)
    for a, b in zip(tuned._trees, ref._trees):
        np.testing.assert_array_equal(a.left_children, b.left_children)
        np.testing.assert_array_equal(a.feature_threshold_array, b.feature_threshold_array)
        np.testing.assert_array_equal(a.values_array, b.values_array)
    plain = RandomForestClassifier(n_estimators=3, seed=5, fit_mode="plain").autotune(x, y, sample_trees=2)
    assert plain["bfs_threshold"] >= 2


def test_many_classes_use_16_bit_labels(cuda_device):
    """More than 255 classes: 2-byte labels through every kernel (level
    steps and warp subtrees), against the oracle."""
    rng = np.random.default_rng(40)
    n = 3000
    y = rng.integers(0, 300, size=n) * 7  # 300 distinct, non-contiguous labels
    x = (rng.normal(size=(n, 10)) + (y[:, None] % 13) * 0.3).astype(np.float32)
    forest = RandomForestClassifier(n_estimators=3, seed=41).fit(x, y)
    assert forest.dtype_labels == np.uint16
    ref = O.fit_forest(x, y, n_estimators=3, seed=41)
    _assert_same_trees(forest._trees, ref.trees)
    np.testing.assert_array_equal(forest.predict(x[:500]), O.predict(ref, x[:500]))


@pytest.mark.parametrize("case", ["one_row", "two_rows_same", "one_feature", "constant_features",
                                  "large_mss", "all_features"])
def test_edge_shapes_match_oracle(cuda_device, case):
    rng = np.random.default_rng(50)
    kw = {}
    if case == "one_row":
        x, y = np.array([[1.0, 2.0]], np.float32), np.array([3])
    elif case == "two_rows_same":
        x, y = np.array([[1.0], [2.0]], np.float32), np.array([5, 5])
    elif case == "one_feature":
        x = rng.normal(size=(700, 1)).astype(np.float32)
        y = (x[:, 0] > 0.2).astype(np.int64) + rng.integers(0, 2, 700)
    elif case == "constant_features":
        x = rng.normal(size=(600, 6)).astype(np.float32)
        x[:, [0, 2, 5]] = 4.0
        y = rng.integers(0, 3, 600)
    elif case == "large_mss":
        x, y = _synthetic(900, 8, 4, 51)
        kw = {"min_samples_split": 60}
    else:
        x, y = _synthetic(900, 8, 4, 52)
        kw = {"max_features": 8}
    forest = RandomForestClassifier(n_estimators=3, seed=53, **kw).fit(x, y)
    ref = O.fit_forest(x, y, n_estimators=3, seed=53, **kw)
    _assert_same_trees(forest._trees, ref.trees)
    np.testing.assert_array_equal(forest.predict(x), O.predict(ref, x))


def test_per_tree_loop_of_hybridforest(cuda_device):
    """The per-tree calls hybridforest's GPU worker makes (fit_init,
    _get_sorted_indices, RandomClassifierTree(forest).fit, fit_release) grow
    the trees a whole-forest fit with the same seed grows."""
    from cudatree_b200 import RandomClassifierTree
    x, y = _synthetic(2500, 9, 4, 61)
    forest = RandomForestClassifier(n_estimators=1, seed=62)
    forest.fit_init(x, y)
    trees = []
    for _ in range(3):
        tree = RandomClassifierTree(forest)
        si, n_samples = forest._get_sorted_indices(forest.sorted_indices)
        tree.fit(forest.samples, forest.target, si, n_samples)
        trees.append(tree)
    forest.fit_release()
    whole = RandomForestClassifier(n_estimators=3, seed=62).fit(x, y)
    for a, b in zip(trees, whole._trees):
        np.testing.assert_array_equal(a.left_children, b.left_children)
        np.testing.assert_array_equal(a.feature_threshold_array, b.feature_threshold_array)
        np.testing.assert_array_equal(a.values_array, b.values_array)


def _two_valued_data(n, c, seed):
    """Two-valued features of every kind the boundary search meets, beside
    continuous ones: {0, 1}; {-0.0, +0.0, 3.5} (two values: -0.0 == +0.0);
    {1, 1 + 4e-6} (never a candidate: closer than 1e-5); {-2, 7.25} tied to
    the class; and one constant feature."""
    rng = np.random.default_rng(seed)
    y = rng.integers(0, c, size=n)
    x = np.zeros((n, 9), np.float32)
    x[:, 0] = rng.normal(size=n) + y
    x[:, 1] = rng.integers(0, 2, n)
    x[:, 2] = np.where(rng.random(n) < 0.5, np.where(rng.random(n) < 0.5, -0.0, 0.0), 3.5)
    x[:, 3] = np.where(rng.random(n) < 0.4, 1.0, np.float32(1.0 + 4e-6))
    x[:, 4] = np.where((y % 2 == 0) ^ (rng.random(n) < 0.1), -2.0, 7.25)
    x[:, 5] = 4.0
    x[:, 6] = rng.normal(size=n)
    x[:, 7] = (rng.random(n) < 0.03).astype(np.float32)
    x[:, 8] = np.where(y == 0, 1.0, rng.integers(0, 2, n))
    return x, y


@pytest.mark.parametrize("mode", ["plain", "batched"])
@pytest.mark.parametrize("n,c,piece", [(700, 3, None), (9000, 5, None), (9000, 12, 1024), (70000, 7, 4096)])
def test_two_valued_features_match_oracle(cuda_device, n, c, piece, mode):
    """Features with at most two distinct values take the boundary search
    (k_scan_two_valued) instead of the full scan; single- and multi-piece
    nodes, byte-packed (C <= 8) and match (C > 8) class counts, uint16 and
    uint32 entries grow the oracle's trees."""
    x, y = _two_valued_data(n, c, 17)
    forest = RandomForestClassifier(n_estimators=3, max_features=4, seed=29, fit_mode=mode)
    if piece:
        forest._tuned = {"scan_piece": piece, "subtree_cutoff": 32}
    forest.fit(x, y, bfs_threshold=2000)
    ref = O.fit_forest(x, y, n_estimators=3, max_features=4, seed=29)
    _assert_same_trees(forest._trees, ref.trees)
    np.testing.assert_array_equal(forest.predict(x), O.predict(ref, x))


@pytest.mark.parametrize("step_nodes", [0, 7])
@pytest.mark.parametrize("cut", [32, 128])
def test_graph_level_loop_matches_host_loop_and_oracle(cuda_device, step_nodes, cut):
    """The batched form runs its levels of at most graph_samples samples as
    one CUDA graph (a device-side loop condition over persistent launches)
    and larger levels from the host.  Every level in the graph, a switch
    after the first levels, and the host-driven loop throughout all grow the
    oracle's trees; with 7 nodes per step a level takes many steps and the
    warp-subtree list (two steps' worth) overflows into the level steps."""
    x, y = _synthetic(5000, 10, 6, 41)
    ref = O.fit_forest(x, y, n_estimators=5, seed=43)
    for host, graph_samples in ((False, 0xFFFFFFFF), (False, 3000), (True, 0)):
        f = RandomForestClassifier(n_estimators=5, seed=43, subtree_cutoff=cut)
        f.host_level_loop = host
        f.step_nodes = step_nodes
        f.graph_samples = graph_samples
        f.fit(x, y)
        _assert_same_trees(f._trees, ref.trees)
        st = f.last_fit_stats
        assert st["steps"] >= 10 and st["total_launches"] > 0


def test_graph_level_loop_reused_across_fits(cuda_device):
    """Fits of the same shape reuse the instantiated loop graph; a fit of
    another shape builds a new one; the trees stay the oracle's."""
    for n, seed in ((3000, 1), (3000, 2), (4100, 3), (3000, 4)):
        x, y = _synthetic(n, 8, 4, seed)
        f = RandomForestClassifier(n_estimators=3, seed=seed).fit(x, y)
        _assert_same_trees(f._trees, O.fit_forest(x, y, n_estimators=3, seed=seed).trees)


@pytest.mark.parametrize("mode", ["plain", "batched"])
@pytest.mark.parametrize("n,seed", [(3000, 71), (40000, 72), (70000, 73)])
def test_virtual_two_valued_features_match_oracle(cuda_device, n, seed, mode):
    """Covtype-shaped data (44 of 54 features one-hot): with label-carrying
    entries every two-valued feature but feature 0 keeps no index lists (a
    row-order list per node and a value bit per row stand for them).  Those
    fits, the fits that keep every list, and the oracle grow the same trees.
    3,000 rows (16-bit entries) and 70,000 rows (32-bit) carry labels in
    their entries; at 40,000 rows a 16-bit entry holds the row id alone, so
    that fit keeps every list either way."""
    from cudatree_b200 import synthetic
    x, y = synthetic.covtype_like(n=n, seed=seed)
    ref = O.fit_forest(x, y, n_estimators=3, max_features=7, seed=seed)
    for virt in (True, False):
        f = RandomForestClassifier(n_estimators=3, max_features=7, seed=seed, fit_mode=mode)
        f.virtual_features = virt
        f.fit(x, y)
        _assert_same_trees(f._trees, ref.trees)
    np.testing.assert_array_equal(f.predict(x[:3000]), O.predict(ref, x[:3000]))


@pytest.mark.parametrize("f", [65, 130, 300])
def test_constant_feature_masks_beyond_64_features_match_oracle(cuda_device, f):
    """The batched fit keeps one constant-feature mask word per 64 features
    for every node when at least one feature in eight is two-valued:
    features that are constant from the start (some above index 64) and
    few-valued features that turn constant deeper in the tree are skipped by
    the partition and the selection, and the trees are the oracle's."""
    rng = np.random.default_rng(f)
    n = 2500
    y = rng.integers(0, 4, size=n)
    x = (rng.normal(size=(n, f)) + 0.8 * y[:, None] * (np.arange(f) % 5 == 0)).astype(np.float32)
    x[:, 1::4] = rng.integers(0, 2, size=(n, len(range(1, f, 4))))  # two values: constant in many nodes
    x[:, 3::8] = rng.integers(0, 3, size=(n, len(range(3, f, 8))))  # three values
    for j in (2, 64, f - 1):
        x[:, j] = 7.0
    ref = O.fit_forest(x, y, n_estimators=3, max_features=9, seed=f)
    forest = RandomForestClassifier(n_estimators=3, max_features=9, seed=f, fit_mode="batched").fit(x, y)
    _assert_same_trees(forest._trees, ref.trees)
    np.testing.assert_array_equal(forest.predict(x[:500]), O.predict(ref, x[:500]))


@pytest.mark.parametrize("n,f,c", [(70000, 6, 5), (30000, 7, 3)])
def test_partition_shapes_grow_the_same_trees(cuda_device, n, f, c):
    """Every partition shape (CT_PART_*), huge-segment threshold and
    small-segment cutoff the autotuner picks among grows the same trees:
    70,000 rows take 32-bit entries, 30,000 rows 16-bit ones."""
    x, y = _synthetic(n, f, c, 61)
    ref = RandomForestClassifier(n_estimators=3, seed=61).fit(x, y)
    options = [(s, h, 0) for s in range(4) for h in (0, 16384, 0xFFFFFFFF)]
    options += [(0, 0, 1024), (1, 16384, 2048), (2, 0, 4096), (0, 0xFFFFFFFF, 65536)]
    for shape, huge, small in options:
        g = RandomForestClassifier(n_estimators=3, seed=61)
        g._tuned = {"part_shape": shape, "huge_rows": huge, "small_rows": small}
        g.fit(x, y)
        for a, b in zip(g._trees, ref._trees):
            np.testing.assert_array_equal(a.left_children, b.left_children)
            np.testing.assert_array_equal(a.feature_idx_array, b.feature_idx_array)
            np.testing.assert_array_equal(a.feature_threshold_array, b.feature_threshold_array)
            np.testing.assert_array_equal(a.values_array, b.values_array)
    _assert_same_trees(ref._trees, O.fit_forest(x, y, n_estimators=3, seed=61).trees)
