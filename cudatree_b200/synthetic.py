"""Seeded synthetic stand-ins for the benchmark workloads.

The reference benchmarks on scikit-learn digits and covtype
(``benchmark/benchmark_all.py``); covtype is not available offline, so these
generators reproduce the shapes, value types and class structure instead:

* ``digits_like``  1,797 x 64 float32 integers 0-16, 10 balanced classes,
  feature ~ Binomial(16, p[c, f]) with p ~ U(0.05, 0.95)            (seed 1)
* ``covtype_like`` 581,012 x 54 float32: 10 class-conditional Gaussian
  features (means U(-3, 3), sigma U(0.5, 2)), a 4-way and a 40-way one-hot
  group drawn per class, 7 classes with priors
  36.5/48.8/6.2/0.5/1.6/3.0/3.5 %                                    (seed 2)
* ``wide``         10,000 x 3,000 N(0, 1), 50 informative features shifted
  by class means ~ N(0, 1.5), 100 uniform classes                    (seed 3)
* ``blob_job``     one job of the forest queue: n log-uniform in
  [500, 50,000], F uniform in [16, 512], C uniform in [2, 50], Gaussian blobs
  with class-shifted means                                           (seed 4 + job)
"""
from __future__ import annotations

import numpy as np

COVTYPE_PRIORS = np.array([36.5, 48.8, 6.2, 0.5, 1.6, 3.0, 3.5])


def digits_like(n: int = 1797, f: int = 64, c: int = 10, seed: int = 1):
    rng = np.random.default_rng(seed)
    p = rng.uniform(0.05, 0.95, size=(c, f))
    y = np.arange(n) % c
    rng.shuffle(y)
    x = rng.binomial(16, p[y]).astype(np.float32)
    return x, y.astype(np.int64)


def covtype_like(n: int = 581012, seed: int = 2):
    rng = np.random.default_rng(seed)
    c = COVTYPE_PRIORS.shape[0]
    y = rng.choice(c, size=n, p=COVTYPE_PRIORS / COVTYPE_PRIORS.sum())
    mu = rng.uniform(-3.0, 3.0, size=(c, 10))
    sd = rng.uniform(0.5, 2.0, size=(c, 10))
    x = np.zeros((n, 54), dtype=np.float32)
    x[:, :10] = (mu[y] + sd[y] * rng.standard_normal((n, 10))).astype(np.float32)
    for lo, k in ((10, 4), (14, 40)):
        probs = rng.dirichlet(np.full(k, 0.5), size=c)
        cum = np.cumsum(probs, axis=1)
        u = rng.random(n)
        cat = (u[:, None] > cum[y]).sum(axis=1)
        cat = np.minimum(cat, k - 1)
        x[np.arange(n), lo + cat] = 1.0
    return x, y.astype(np.int64)


def wide(n: int = 10000, f: int = 3000, c: int = 100, informative: int = 50, seed: int = 3):
    rng = np.random.default_rng(seed)
    y = rng.integers(0, c, size=n)
    x = rng.standard_normal((n, f)).astype(np.float32)
    cols = rng.choice(f, size=informative, replace=False)
    means = rng.normal(0.0, 1.5, size=(c, informative)).astype(np.float32)
    x[:, cols] += means[y]
    return x, y.astype(np.int64)


def blob_job(job: int):
    rng = np.random.default_rng(4 + job)
    n = int(np.exp(rng.uniform(np.log(500), np.log(50000))))
    f = int(rng.integers(16, 513))
    c = int(rng.integers(2, 51))
    y = rng.integers(0, c, size=n)
    means = rng.normal(0.0, 1.0, size=(c, f)).astype(np.float32)
    x = (rng.standard_normal((n, f)).astype(np.float32) + means[y])
    return x, y.astype(np.int64)
