"""The layout-quality measures used by the device quality tests, on the CPU.

tests/helpers.trustworthiness_torch evaluates trustworthiness with torch so
that 10^4 queries over 10^6 points are affordable on a GPU; here it is checked
to equal the oracle's C implementation (oracle.trustworthiness) exactly on
small inputs, with sampled and full query sets and with duplicate points
(distance ties broken by index).
"""
import numpy as np
import pytest

import oracle
from helpers import trustworthiness_torch

pytest.importorskip("torch")


@pytest.mark.parametrize("n,dim,sample", [(500, 10, 200), (3000, 10, 300), (800, 4, None)])
def test_trustworthiness_torch_equals_oracle(n, dim, sample):
    rng = np.random.default_rng(n + dim)
    X = rng.normal(size=(n, dim))
    X[n // 2:n // 2 + 40] = X[:40]                       # exact duplicates: ties in X
    Y = (X[:, :2] + rng.normal(size=(n, 2)) * 0.5).astype(np.float32)
    q = None if sample is None else np.sort(rng.choice(n, size=sample, replace=False)).astype(np.int32)
    a = oracle.trustworthiness(X, Y, 15, queries=q)
    b = trustworthiness_torch(X, Y, 15, queries=q, device="cpu", batch=64)
    assert a == b, (a, b)


def test_oracle_knn_rows_equals_full_search():
    """The threaded, row-sampled oracle search used at the benchmark sizes
    returns exactly the full search's rows."""
    from helpers import oracle_knn_rows, sampled_rows

    X = oracle.gaussian_mixture(3000, 12, 5, 3.0, seed=4, dtype=np.float32)
    rows = sampled_rows(3000, 4, 50, seed=1)
    idx, dist = oracle_knn_rows(X, 10, rows, 50)
    fidx, fdist = oracle.knn(X, 10)
    assert np.array_equal(idx, fidx[rows]) and np.array_equal(dist, fdist[rows])
