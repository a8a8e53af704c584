"""Seeded inputs shaped like the reference's test fixtures (tests/src/*.cpp).

The reference draws its fixtures from std::mt19937_64 through knncolle and
aarand (absent here); these generators use NumPy's PCG64 with the same shapes
and distributions, and the exact kNN of the oracle in place of the VP-tree.
"""
from __future__ import annotations

import numpy as np

import oracle


def normal_data(n: int, dim: int, seed: int, dtype=np.float64) -> np.ndarray:
    """iid N(0, 1) data (tests/src/neighbor_similarities.cpp:14-22)."""
    return np.random.default_rng(seed).normal(size=(n, dim)).astype(dtype)


def two_populations(n: int, dim: int, seed: int, dtype=np.float64) -> np.ndarray:
    """U(0, 1) data with odd observations shifted by 10 on dimension 0 (tests/src/umappp.cpp:18-33)."""
    x = np.random.default_rng(seed).uniform(size=(n, dim))
    x[1::2, 0] += 10
    return x.astype(dtype)


def neighbors_of(data: np.ndarray, k: int, dtype=None) -> oracle.CSR:
    """Exact kNN as a CSR NeighborList (distances in the data's type unless dtype is given)."""
    idx, dist = oracle.knn(data, k)
    return oracle.CSR.from_dense(idx, dist.astype(dtype or data.dtype))


def mock_probabilities(n: int, seed: int) -> oracle.CSR:
    """Random symmetric weighted graph with a forced chain, hence connected
    (tests/src/spectral_init.cpp:14-34)."""
    rng = np.random.default_rng(seed)
    rows = [[] for _ in range(n)]
    for r in range(n):
        forced = (n if r == 0 else r) - 1
        for c in range(r):
            if c == forced or rng.uniform() < 0.2:
                v = rng.uniform()
                rows[r].append((c, v))
                rows[c].append((r, v))
    rows = [sorted(r) for r in rows]
    return oracle.CSR.from_lists(rows)


def mock_neighbors(n: int, k: int, seed: int) -> oracle.CSR:
    """Random neighbour lists with increasing distances and a forced link to the
    previous observation (tests/src/umappp.cpp:175-205)."""
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        forced = (n if i == 0 else i) - 1
        cand = rng.choice(np.setdiff1d(np.arange(n), [i]), size=k, replace=False)
        if forced not in cand:
            cand[0] = forced
        rng.shuffle(cand)
        d = np.cumsum(rng.uniform(size=k))
        rows.append(list(zip(cand.tolist(), d.tolist())))
    return oracle.CSR.from_lists(rows)


def csr_tuple(g: oracle.CSR):
    return g.ptr, g.idx, g.val


def rel_err(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.maximum(np.abs(b), 1e-300)
    return float(np.max(np.abs(a - b) / den)) if a.size else 0.0


def eigen_check(g: oracle.CSR, Y: np.ndarray, tol: float = 1e-4) -> bool:
    """The reference's eigen-equation check (tests/src/spectral_init.cpp:36-85):
    (I - D^-1/2 W D^-1/2) y is proportional to y for every output column."""
    n, ndim = Y.shape
    sums = np.sqrt(np.array([g.val[g.ptr[i]:g.ptr[i + 1]].sum() for i in range(n)], dtype=np.float64))
    out = Y.astype(np.float64).copy()
    for o in range(n):
        for p in range(g.ptr[o], g.ptr[o + 1]):
            j = g.idx[p]
            out[o] += Y[j] * (-g.val[p] / sums[o] / sums[j])
    res_scale = Y.astype(np.float64).sum(axis=0)
    copy_scale = out.sum(axis=0)
    ref = Y.astype(np.float64)
    cmp = out * res_scale / copy_scale
    return bool(np.all(np.abs(ref - cmp) < tol * (np.abs(ref) + np.abs(cmp)) / 2 + 1e-12))
