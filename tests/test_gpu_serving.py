"""Serving engine: each request's predictions equal the plain predict path,
alone and inside a mixed replay of concurrent requests of different sizes and
forests; a fit job through the server yields the same forest as the Python
fit with the same seed; admission rejects work that does not fit."""
import numpy as np
import pytest
import torch
from sklearn.datasets import load_digits, load_iris

from cudatree_b200 import CudaTreeError, RandomForestClassifier
from cudatree_b200.serving import ForestServer, pinned

pytestmark = pytest.mark.gpu


def _blobs(n, f, c, seed):
    rng = np.random.default_rng(seed)
    y = rng.integers(0, c, size=n)
    means = rng.normal(scale=1.5, size=(c, f))
    return (rng.normal(size=(n, f)) + means[y]).astype(np.float32), y


@pytest.fixture(scope="module")
def served(cuda_device):
    xa, ya = load_digits().data.astype(np.float32), load_digits().target
    xb, yb = _blobs(4000, 37, 9, 3)
    fa = RandomForestClassifier(n_estimators=40, seed=1).fit(xa, ya)
    fb = RandomForestClassifier(n_estimators=25, seed=2).fit(xb, yb)
    srv = ForestServer(max_features=64, fit_workers=1, max_fit_rows=5000, max_fit_trees=8)
    ida, idb = srv.add_forest(fa), srv.add_forest(fb)
    yield srv, [(ida, fa, xa), (idb, fb, xb)]
    srv.close()


def test_single_requests_match_plain_predict(served):
    srv, forests = served
    for fid, forest, x in forests:
        for n in (1, 7, 300, x.shape[0]):
            np.testing.assert_array_equal(srv.predict(fid, x[:n]), forest.predict(x[:n]))


def test_mixed_replay_matches_plain_predict(served):
    srv, forests = served
    rng = np.random.default_rng(7)
    reqs, keep = [], []
    t = 0.0
    for i in range(200):
        fid, forest, x = forests[i % 2]
        n = int(np.exp(rng.uniform(0, np.log(x.shape[0]))))
        lo = int(rng.integers(0, x.shape[0] - n + 1))
        xp = pinned(x[lo:lo + n])
        out = torch.zeros(n, dtype=torch.int32).pin_memory()
        r = srv.predict_request(fid, xp, out)
        t += rng.exponential(1 / 4000.0)
        r.arrival_s = t
        reqs.append(r)
        keep.append((forest, x[lo:lo + n], xp, out))
    stats = srv.replay(reqs)
    assert stats["requests"] == 200 and stats["rejected"] == 0
    assert stats["p99_ms"] >= stats["p50_ms"] > 0
    assert stats["zero_copy_requests"] > 0  # small requests on pinned buffers skip the copies
    for r, (forest, xs, xp, out) in zip(reqs, keep):
        assert r.status == 0
        got = forest.compt_table[out.numpy().astype(np.int64)]
        np.testing.assert_array_equal(got, forest.predict(xs))


def test_fit_job_matches_python_fit(served):
    srv, _ = served
    x, y = _blobs(3000, 20, 6, 11)
    xp, yp = pinned(x), pinned(y.astype(np.uint32))
    req = srv.fit_request(xp, yp, n_classes=6, n_trees=5, seed=99, max_features=4)
    srv.submit(req)
    assert srv.wait(req) == 0
    ref = RandomForestClassifier(n_estimators=5, max_features=4, seed=99).fit(x, y)
    np.testing.assert_array_equal(srv.predict(req.result_forest, x), ref.predict(x))


def test_admission_rejects_oversize(served):
    srv, forests = served
    fid, forest, x = forests[1]
    big = np.zeros((200000, forest.n_features), dtype=np.float32)
    with pytest.raises(CudaTreeError):
        srv.predict(fid, big)
    x2, y2 = _blobs(20000, 64, 3, 5)  # 4x the rows the fit arena was sized for
    req = srv.fit_request(pinned(x2), pinned(y2.astype(np.uint32)), n_classes=3, n_trees=8, seed=1)
    srv.submit(req)
    assert srv.wait(req) == 2  # CT_ERR_OOM


def test_budget_too_small_fails_cleanly(cuda_device):
    with pytest.raises(CudaTreeError):
        ForestServer(hbm_budget_bytes=1 << 20)


def test_tree_groups_match_oracle_and_server(cuda_device):
    """Large trees (noise labels, fully grown) split the forest into several
    L2-sized tree groups; grouped votes must equal the oracle's votes, and
    the server's batched path must equal the plain path."""
    from oracle import cudatree_oracle as O
    rng = np.random.default_rng(4)
    x = rng.normal(size=(200000, 8)).astype(np.float32)
    y = rng.integers(0, 5, size=200000)
    forest = RandomForestClassifier(n_estimators=40, seed=8).fit(x, y)
    per_tree = sum(t.n_nodes for t in forest._trees) * 16 / 40
    assert 32 * 2**20 / per_tree < 40, "test forest must need several tree groups"
    xs = x[:3000]
    ref = O.Forest(trees=[O.Tree(t.left_children, t.right_children, t.feature_idx_array,
                                 t.feature_threshold_array, t.values_array.astype(np.int64))
                          for t in forest._trees], classes=forest.compt_table, n_features=8)
    np.testing.assert_array_equal(forest.predict(xs), O.predict(ref, xs))
    np.testing.assert_array_equal(forest.predict_proba(xs), O.predict_proba(ref, xs))
    srv = ForestServer(max_features=16, fit_workers=0)
    fid = srv.add_forest(forest)
    small = RandomForestClassifier(n_estimators=20, seed=9).fit(x[:5000], y[:5000])
    sid = srv.add_forest(small)
    reqs, keep = [], []
    for i, n in enumerate([1, 2000, 37, 5000, 4096, 9000, 3]):
        f, fi = (forest, fid) if i % 2 == 0 else (small, sid)
        xp = pinned(x[i * 10000:i * 10000 + n])
        out = torch.zeros(n, dtype=torch.int32).pin_memory()
        r = srv.predict_request(fi, xp, out)
        r.arrival_s = 0.0
        reqs.append(r)
        keep.append((f, x[i * 10000:i * 10000 + n], out, xp))  # buffers live until completion
    srv.replay(reqs)
    for r, (f, xs2, out, _) in zip(reqs, keep):
        assert r.status == 0
        np.testing.assert_array_equal(f.compt_table[out.numpy().astype(np.int64)], f.predict(xs2))
    srv.close()


def test_forest_pool_remove_and_reuse(cuda_device):
    """Forests live in a pool reserved at creation: a forest larger than the
    pool is refused, a removed forest's bytes are reused, and requests for a
    removed forest fail."""
    x, y = _blobs(3000, 12, 4, 21)
    forest = RandomForestClassifier(n_estimators=12, seed=3).fit(x, y)
    assert forest._compact_fits()  # held as 8-byte nodes

    def up(b):
        return (b + 255) // 256 * 256
    need = up(up(8 * sum(t.n_nodes for t in forest._trees)) + 4 * len(forest._trees))
    srv = ForestServer(max_features=16, fit_workers=0, forest_pool_bytes=int(need * 1.5))
    a = srv.add_forest(forest)
    with pytest.raises(CudaTreeError):
        srv.add_forest(forest)  # the pool holds one copy
    assert srv.stats()["forest_bytes"] == need
    srv.remove_forest(a)
    assert srv.stats()["forest_bytes"] == 0
    with pytest.raises(CudaTreeError):
        srv.predict(a, x[:10])
    b = srv.add_forest(forest)
    np.testing.assert_array_equal(srv.predict(b, x), forest.predict(x))
    srv.close()


def _same_trees(a, b):
    assert len(a._trees) == len(b._trees)
    for s, t in zip(a._trees, b._trees):
        np.testing.assert_array_equal(s.left_children, t.left_children)
        np.testing.assert_array_equal(s.right_children, t.right_children)
        np.testing.assert_array_equal(s.feature_idx_array, t.feature_idx_array)
        np.testing.assert_array_equal(s.feature_threshold_array, t.feature_threshold_array)
        np.testing.assert_array_equal(s.values_array.astype(np.int64), t.values_array.astype(np.int64))


def test_read_forest_round_trip(served):
    srv, forests = served
    for fid, forest, x in forests:
        back = srv.forest(fid)
        _same_trees(back, forest)
        np.testing.assert_array_equal(back.predict(x[:500]), forest.predict(x[:500]))


def test_forest_queue_matches_solo_fits(cuda_device):
    """Uneven jobs fitted concurrently through the queue give, job by job, the
    trees a solo fit with the same seed gives."""
    from cudatree_b200.serving import fit_forests
    rng = np.random.default_rng(12)
    jobs = []
    for j in range(7):
        n = int(rng.integers(300, 6000))
        f = int(rng.integers(3, 90))
        c = int(rng.integers(2, 12))
        x, y = _blobs(n, f, c, 100 + j)
        jobs.append((x, y * 3 + 1))  # labels that need compaction
    seeds = [1000 + j for j in range(len(jobs))]
    got = fit_forests(jobs, n_estimators=6, seeds=seeds)
    for (x, y), seed, g in zip(jobs, seeds, got):
        solo = RandomForestClassifier(n_estimators=6, seed=seed).fit(x, y)
        _same_trees(g, solo)
        np.testing.assert_array_equal(g.predict(x), solo.predict(x))
