"""Generate the golden fixtures under tests/golden/ (run from the repo root).

    python tests/golden/make_golden.py

* ``reference_chain_nodes.npz`` — seeded random nodes of the iris, digits and
  diabetes data (the datasets of the reference's own tests, bundled with
  scikit-learn) with, for each node, the output of the literal restatement of
  the reference's DFS kernel chain (``oracle.reference_dfs_node_split``:
  imp_left, imp_right, split position, feature slot) next to the canonical
  rule's minimum score.
* ``oracle_forests.npz`` — canonical forests (node arrays in breadth-first
  order) of small seeded fits, which the GPU tests compare node for node and
  the CPU tests use to detect drift of the oracle.
* ``covtype_trees.json`` — node counts and SHA-256 digests of the first
  trees of the oracle forest at the benchmark's full covtype-shaped size
  (581,012 x 54, 7 classes, max_features 7, bootstrap, seed 1000): the GPU
  parity test checks its trees against them, and a CPU test regrows them to
  catch drift of the oracle.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
from sklearn.datasets import load_diabetes, load_digits, load_iris

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from cudatree_b200 import synthetic  # noqa: E402
from oracle import cudatree_oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent


def datasets():
    return {
        "iris": (load_iris().data, load_iris().target),
        "digits": (load_digits().data, load_digits().target),
        "diabetes": (load_diabetes().data, (load_diabetes().target > 140).astype(np.int64)),
    }


def reference_chain_nodes(nodes_per_set: int = 40):
    rng = np.random.default_rng(2024)
    rec = {k: [] for k in ("set", "members_off", "members", "feats_off", "feats", "ref_l", "ref_r",
                           "ref_split", "ref_slot", "canon_score", "canon_feature", "canon_pos")}
    moff, foff = [0], [0]
    names = []
    for si, (name, (x, y)) in enumerate(datasets().items()):
        names.append(name)
        x = np.asarray(x, dtype=np.float32)
        xf = np.ascontiguousarray(x.T)
        c = int(y.max()) + 1
        for _ in range(nodes_per_set):
            n = int(rng.integers(2, x.shape[0] + 1))
            members = np.sort(rng.choice(x.shape[0], n, replace=False))
            feats = list(rng.choice(x.shape[1], min(8, x.shape[1]), replace=False))
            totals = np.bincount(y[members], minlength=c)
            best = None
            for f in sorted(feats):
                order, xs = O.node_sorted(xf, f, members)
                r = O.scan_sorted(xs, y[members[order]], totals)
                if r and (best is None or r[0] < best[0]):
                    best = (r[0], f, r[1])
            lists = [(f, members[O.node_sorted(xf, f, members)[0]]) for f in feats]
            rl, rr, rs, rf = O.reference_dfs_node_split(xf, y, lists, c)
            rec["set"].append(si)
            rec["members"].extend(members.tolist())
            moff.append(moff[-1] + n)
            rec["feats"].extend(int(f) for f in feats)
            foff.append(foff[-1] + len(feats))
            rec["ref_l"].append(np.float32(rl))
            rec["ref_r"].append(np.float32(rr))
            rec["ref_split"].append(int(rs))
            rec["ref_slot"].append(int(rf))
            rec["canon_score"].append(best[0] if best else np.inf)
            rec["canon_feature"].append(best[1] if best else -1)
            rec["canon_pos"].append(best[2] if best else -1)
    np.savez_compressed(
        OUT / "reference_chain_nodes.npz", names=np.array(names), set=np.array(rec["set"]),
        members=np.array(rec["members"], np.int32), members_off=np.array(moff, np.int64),
        feats=np.array(rec["feats"], np.int32), feats_off=np.array(foff, np.int64),
        ref_l=np.array(rec["ref_l"], np.float32), ref_r=np.array(rec["ref_r"], np.float32),
        ref_split=np.array(rec["ref_split"], np.int64), ref_slot=np.array(rec["ref_slot"], np.int64),
        canon_score=np.array(rec["canon_score"]), canon_feature=np.array(rec["canon_feature"]),
        canon_pos=np.array(rec["canon_pos"]))


FOREST_CASES = {
    # name: (data builder, n_estimators, bootstrap, max_features, seed)
    "iris_nobs": (lambda: (load_iris().data, load_iris().target), 3, False, None, 123),
    "digits_like_nobs": (lambda: synthetic.digits_like(), 2, False, 8, 11),
    "digits_bs": (lambda: (load_digits().data, load_digits().target), 2, True, None, 5),
}


def oracle_forests():
    arrays = {}
    for name, (make, t, bs, m, seed) in FOREST_CASES.items():
        x, y = make()
        f = O.fit_forest(x, y, n_estimators=t, bootstrap=bs, max_features=m, seed=seed)
        for i, tr in enumerate(f.trees):
            for field in ("left", "right", "feature", "threshold", "value"):
                arrays[f"{name}/{i}/{field}"] = getattr(tr, field)
    np.savez_compressed(OUT / "oracle_forests.npz", **arrays)


COVTYPE = {"make": "covtype_like", "seed": 1000, "max_features": 7, "bootstrap": True, "trees": 3}


def covtype_trees():
    import json

    from tests import oracle_jobs
    c = COVTYPE
    with oracle_jobs.pool(c["trees"]) as ex:
        trees = [f.result() for f in oracle_jobs.submit_forest(ex, c["make"], None, c["trees"], c["seed"],
                                                                c["max_features"], c["bootstrap"])]
    rec = dict(c, workload="covtype-shaped synthetic 581012x54 f32, 7 classes",
               digests=[{"tree": i, "n_nodes": t.n_nodes, "sha256": oracle_jobs.oracle_digest(t)}
                        for i, t in enumerate(trees)])
    (OUT / "covtype_trees.json").write_text(json.dumps(rec, indent=1) + "\n")


if __name__ == "__main__":
    reference_chain_nodes()
    oracle_forests()
    covtype_trees()
    for p in sorted(OUT.glob("*.npz")):
        print(p.name, p.stat().st_size, "bytes")
