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


def same_neighbors(idx_a, idx_b, dist_ref, rel_tie=1e-6) -> int:
    """Number of neighbour positions where idx_a differs from idx_b other than
    by an exchange of (near-)tied reference distances (within rel_tie)."""
    bad = 0
    for i in range(idx_a.shape[0]):
        if np.array_equal(idx_a[i], idx_b[i]):
            continue
        d = dist_ref[i]
        for c in np.nonzero(idx_a[i] != idx_b[i])[0]:
            lo = max(c - 1, 0)
            hi = min(c + 1, len(d) - 1)
            near = np.abs(d[lo:hi + 1] - d[c]) <= rel_tie * max(d[c], 1e-300)
            if near.sum() < 2:
                bad += 1
    return bad


def sampled_rows(n: int, blocks: int, block_len: int, seed: int) -> np.ndarray:
    """blocks non-overlapping runs of block_len consecutive rows at seeded
    random offsets (sorted)."""
    rng = np.random.default_rng(seed)
    span = n // blocks
    starts = [b * span + int(rng.integers(0, max(span - block_len, 1))) for b in range(blocks)]
    return np.concatenate([np.arange(s, min(s + block_len, n)) for s in starts])


def oracle_knn_rows(X: np.ndarray, k: int, rows: np.ndarray, block_len: int, threads: int = 0):
    """The oracle's exact FP64 kNN (oracle.knn) of the given rows, which come
    in runs of block_len consecutive rows (sampled_rows); the runs are searched
    in parallel host threads (the C search releases the GIL)."""
    import concurrent.futures
    import os

    X64 = np.ascontiguousarray(X, dtype=np.float64)   # what oracle_knn_f32 would convert to
    starts = rows[::block_len]
    threads = threads or min(len(starts), os.cpu_count() or 1)
    with concurrent.futures.ThreadPoolExecutor(threads) as ex:
        parts = list(ex.map(lambda s: oracle.knn(X64, k, int(s), int(min(block_len, X.shape[0] - s))), starts))
    return np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts])


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


def trustworthiness_torch(X: np.ndarray, Y: np.ndarray, k: int = 15, queries: np.ndarray | None = None,
                          device: str = "cuda", batch: int = 8) -> float:
    """Trustworthiness(k) of embedding Y for data X, as oracle.trustworthiness
    computes it (FP64 squared distances, ranks with ties broken by index,
    queries optionally a sample of rows; sklearn.manifold.trustworthiness's
    formula), evaluated with torch on 'device' so that 10^4 queries against
    10^6 points take seconds.  Test infrastructure: a quality measure of
    layouts, not a stage of the product."""
    import torch

    n = X.shape[0]
    q = np.arange(n) if queries is None else np.asarray(queries)
    Xd = torch.as_tensor(np.ascontiguousarray(X), device=device).to(torch.float64)
    Yd = torch.as_tensor(np.ascontiguousarray(Y), device=device).to(torch.float64)
    ar = torch.arange(n, device=device)
    total = 0.0
    for s in range(0, len(q), batch):
        qi = torch.as_tensor(q[s:s + batch], device=device, dtype=torch.long)
        rows = torch.arange(len(qi), device=device)
        dX = ((Xd[None, :, :] - Xd[qi][:, None, :]) ** 2).sum(-1)          # (b, n)
        dY = ((Yd[None, :, :] - Yd[qi][:, None, :]) ** 2).sum(-1)
        dY[rows, qi] = float("inf")
        # k nearest in Y, ties by index: among the k + 8 smallest, sort by (distance, index)
        cand = torch.topk(dY, min(k + 8, n - 1), dim=1, largest=False).indices
        cand = torch.sort(cand, dim=1).values
        cd = torch.gather(dY, 1, cand)
        order = torch.argsort(cd, dim=1, stable=True)
        nb = torch.gather(cand, 1, order)[:, :k]                            # (b, k)
        dj = torch.gather(dX, 1, nb)                                        # (b, k)
        for t in range(k):
            d = dj[:, t:t + 1]
            j = nb[:, t:t + 1]
            closer = (dX < d) | ((dX == d) & (ar[None, :] < j))
            closer[rows, qi] = False
            rank = closer.sum(1) + 1                                        # j itself is never 'closer'
            total += float(torch.clamp(rank - k, min=0).sum())
    return 1.0 - 2.0 / (len(q) * k * (2.0 * n - 3.0 * k - 1.0)) * total
