"""CPU checks of the oracle: the reference's known-answer tests, agreement
with the literal restatement of the reference's DFS kernel chain (committed
fixtures), drift against the committed canonical forests, and the RNG
building blocks."""
from pathlib import Path

import numpy as np
import pytest
from sklearn.datasets import load_diabetes, load_digits, load_iris

from oracle import cudatree_oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"


def _sets():
    return {
        "iris": (load_iris().data, load_iris().target),
        "digits": (load_digits().data, load_digits().target),
        "diabetes": (load_diabetes().data, (load_diabetes().target > 140).astype(np.int64)),
    }


@pytest.mark.parametrize("name", ["iris", "digits", "diabetes"])
def test_memorize_known_answer(name):
    """test/test_iris.py:7-14, test/test_digits.py:10-17, test/test_diabetes_classify.py:7-14."""
    x, y = _sets()[name]
    forest = O.fit_forest(x, y, n_estimators=3, bootstrap=False, seed=9)
    assert int((O.predict(forest, x) != y).sum()) == 0


def test_canonical_minimum_matches_reference_chain():
    g = np.load(GOLDEN / "reference_chain_nodes.npz")
    sets = _sets()
    names = list(g["names"])
    for i in range(g["set"].shape[0]):
        x, y = sets[names[g["set"][i]]]
        xf = np.ascontiguousarray(np.asarray(x, np.float32).T)
        members = g["members"][g["members_off"][i]:g["members_off"][i + 1]].astype(np.int64)
        feats = g["feats"][g["feats_off"][i]:g["feats_off"][i + 1]]
        c = int(y.max()) + 1
        totals = np.bincount(y[members], minlength=c)
        best = None
        for f in sorted(int(v) for v in feats):
            order, xs = O.node_sorted(xf, f, members)
            r = O.scan_sorted(xs, y[members[order]], totals)
            if r and (best is None or r[0] < best[0]):
                best = (r[0], f, r[1], r[2], r[3])
        ref_sum = float(np.float32(g["ref_l"][i]) + np.float32(g["ref_r"][i]))
        if best is None:
            assert ref_sum == 4.0 and g["canon_feature"][i] == -1
            continue
        # the oracle has not drifted from the committed canonical choice
        assert best[0] == g["canon_score"][i] and best[1] == g["canon_feature"][i] and best[2] == g["canon_pos"][i]
        # the reference chain reaches the same minimum impurity
        assert abs(float(np.float32(best[3]) + np.float32(best[4])) - ref_sum) <= 1e-6
        # and its own choice scores the same minimum in fp64 (a tie, if the choice differs)
        f_ref = int(feats[g["ref_slot"][i]])
        order, xs = O.node_sorted(xf, f_ref, members)
        lab = y[members[order]]
        n = members.shape[0]
        p = int(g["ref_split"][i])
        cnt = np.bincount(lab[: p + 1], minlength=c).astype(np.int64)
        nl, nr = float(p + 1), float(n - p - 1)
        il = (1.0 - float(np.sum(cnt * cnt)) / (nl * nl)) * (nl / n)
        rc = totals - cnt
        ir = (1.0 - float(np.sum(rc * rc)) / (nr * nr)) * (nr / n)
        assert abs((il + ir) - best[0]) <= 1e-6


def test_oracle_reproduces_golden_forests():
    from tests.golden.make_golden import FOREST_CASES
    g = np.load(GOLDEN / "oracle_forests.npz")
    for name, (make, t, bs, m, seed) in FOREST_CASES.items():
        x, y = make()
        f = O.fit_forest(x, y, n_estimators=t, bootstrap=bs, max_features=m, seed=seed)
        for i, tr in enumerate(f.trees):
            for field in ("left", "right", "feature", "threshold", "value"):
                np.testing.assert_array_equal(getattr(tr, field), g[f"{name}/{i}/{field}"], err_msg=f"{name}/{i}/{field}")


@pytest.mark.parametrize("n_features", [1, 2, 3, 4, 5, 7, 54, 64, 100, 513, 3000])
def test_feature_permutation_is_a_bijection(n_features):
    for key in (0, O.mix64(1), O.mix64(2)):
        perm = [O.feature_perm(i, n_features, key) for i in range(n_features)]
        assert sorted(perm) == list(range(n_features))


def test_bootstrap_draws():
    a = O.bootstrap_draws(5, 3, 10000)
    b = O.bootstrap_draws(5, 3, 10000)
    np.testing.assert_array_equal(a, b)
    assert a.min() >= 0 and a.max() < 10000
    frac = np.unique(a).shape[0] / 10000
    assert 0.60 < frac < 0.66   # 1 - 1/e in-bag fraction
    assert not np.array_equal(a, O.bootstrap_draws(5, 4, 10000))
    np.testing.assert_array_equal(O.bootstrap_rows(5, 3, 7, False), np.arange(7))


def test_presort_ties_and_negative_zero():
    x = np.array([[0.0, -0.0, 1.0, -1.0, 0.0, -0.0]], dtype=np.float32)
    np.testing.assert_array_equal(O.presort(x)[0], [3, 0, 1, 4, 5, 2])


def test_accuracy_close_to_sklearn():
    """Pattern of test/helpers.py:4-28 (train on one half, score the other)."""
    from sklearn.ensemble import RandomForestClassifier as SkRF
    x, y = load_digits().data, load_digits().target
    n = x.shape[0] // 2
    ours = O.fit_forest(x[:n], y[:n], n_estimators=8, bootstrap=True, seed=1)
    ours_score = float(np.mean(O.predict(ours, x[n:]) == y[n:]))
    sk = SkRF(n_estimators=8, random_state=0).fit(x[:n], y[:n]).score(x[n:], y[n:])
    assert ours_score >= 0.9 * sk


def test_candidate_shortcut_matches_double_test():
    """The split scan decides 'x + 1e-5 < x_next' (double) with a float
    shortcut: equal values never qualify, a float gap above 1e-4 always does.
    Check the shortcut against the double test on edge and random pairs."""
    rng = np.random.default_rng(0)
    base = np.concatenate([
        rng.normal(size=20000), rng.normal(scale=1e6, size=5000), rng.normal(scale=1e-6, size=5000),
        [0.0, -0.0, 1e-5, -1e-5, 1e-4, 3e38, -3e38, 1e30, 2.0 ** 37, 65504.0]]).astype(np.float32)
    gaps = np.concatenate([
        np.zeros(base.size // 4), rng.uniform(0, 3e-5, base.size // 4),
        rng.uniform(9e-5, 1.1e-4, base.size // 4), rng.exponential(1e-3, base.size - 3 * (base.size // 4))])
    x = base
    xn = (x.astype(np.float64) + gaps.astype(np.float64)).astype(np.float32)
    near = np.nextafter(x, np.float32(np.inf))  # one ulp apart
    x = np.concatenate([x, x, xn]).astype(np.float32)
    xn = np.concatenate([xn, near, x[: xn.size]]).astype(np.float32)  # includes x > x_next pairs
    exact = (x.astype(np.float64) + 1e-5) < xn.astype(np.float64)
    with np.errstate(over="ignore", invalid="ignore"):
        d = (xn - x).astype(np.float32)
    fast = np.where(~(xn > x), False, np.where(d > np.float32(1e-4), True, exact))
    np.testing.assert_array_equal(fast, exact)


def test_covtype_full_size_oracle_trees_match_fixture():
    """The oracle's first three trees of the benchmark forest (581,012 x 54
    covtype-shaped, 7 classes, max_features 7, bootstrap, seed 1000) against
    the node counts and digests committed in tests/golden/covtype_trees.json:
    the GPU parity test pins its trees to the same digests."""
    import json
    from pathlib import Path

    from tests import oracle_jobs
    fx = json.loads((Path(__file__).resolve().parent / "golden" / "covtype_trees.json").read_text())
    with oracle_jobs.pool(fx["trees"]) as ex:
        trees = [f.result() for f in oracle_jobs.submit_forest(ex, fx["make"], None, fx["trees"], fx["seed"],
                                                                fx["max_features"], fx["bootstrap"])]
    for d, t in zip(fx["digests"], trees):
        assert t.n_nodes == d["n_nodes"], d["tree"]
        assert oracle_jobs.oracle_digest(t) == d["sha256"], d["tree"]
