"""Exactness of the device kNN at the benchmark's sizes.

The tensor-core search prunes reference tiles with FP32 bounds carrying
relative safety margins and recomputes in FP64 only the queries whose
candidate list is not provably complete; a wrong bound would drop true
neighbours silently, and most visibly on large, clustered inputs.  Here the
device searches the benchmark data sets in full (100,000 x 50 and
1,000,000 x 50 Gaussian mixtures, k = 15) and 1,000 sampled query rows are
checked against the oracle's exact FP64 brute force over all points: the
neighbour indices must be equal except where reference distances tie within
1e-6 (relative), and the distances must be the FP64 values rounded to float
(1e-6 relative).
"""
import numpy as np
import pytest

import bench
from helpers import oracle_knn_rows, rel_err, same_neighbors, sampled_rows

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("workload", ["mixture_100k", "mixture_1m"])
def test_knn_exact_on_benchmark_data(umap, workload):
    X = bench.make_data(workload)
    k = bench.CONFIGS[workload][5]
    idx, dist = umap.knn(X, k)
    L = umap.lib()
    rows = sampled_rows(X.shape[0], 8, 125, seed=2024)
    ridx, rdist = oracle_knn_rows(X, k, rows, 125)
    bad = same_neighbors(idx[rows], ridx, rdist)
    err = rel_err(dist[rows], rdist)
    print(f"{workload}: {len(rows)} sampled queries, non-tie mismatches {bad}, max distance rel. error {err:.2e}, "
          f"FP64-recomputed queries {L.umapb_knn_last_fp64_recomputed()}, tile pairs {L.umapb_knn_last_tile_pairs()}, "
          f"largest tensor-core distance error {L.umapb_knn_last_tc_error():.2e}")
    assert bad == 0
    assert err <= 1e-6


@pytest.mark.parametrize("workload,dtype,num_shards", [("mixture_100k", np.float32, 2), ("mixture_100k", np.float32, 7),
                                                       ("mixture_100k", np.float64, 3)])
def test_knn_shards_partition_and_reproduce_full_search(umap, workload, dtype, num_shards):
    """umapb_knn_shard: the shards' rows partition the observations and, put
    together, equal the unsharded search bit for bit (indices and distances)."""
    X = bench.make_data(workload).astype(dtype)
    k = bench.CONFIGS[workload][5]
    idx, dist = umap.knn(X, k)
    seen = np.zeros(X.shape[0], np.int64)
    got_idx = np.full_like(idx, -1)
    got_dist = np.zeros_like(dist)
    counts = []
    for s in range(num_shards):
        rows, si, sd = umap.knn_shard(X, k, s, num_shards)
        assert np.all(np.diff(rows) > 0)
        seen[rows] += 1
        got_idx[rows] = si
        got_dist[rows] = sd
        counts.append(len(rows))
    print(f"{workload} {np.dtype(dtype).name} {num_shards} shards: rows per shard {counts}")
    assert np.all(seen == 1)
    assert np.array_equal(got_idx, idx)
    assert np.array_equal(got_dist, dist)


def test_knn_launch_shapes_agree_and_are_exact(umap, monkeypatch):
    """The launch shapes of the FP16 search for dim <= 63 (UMAPB_KNN_SHAPE: 24
    = two query tiles per CTA, 4-stage ring; 12 = one query tile, 2-stage
    ring, two CTAs per SM) give the same lists, equal to the FP64 oracle on
    sampled rows."""
    X = bench.make_data("mixture_100k")
    k = bench.CONFIGS["mixture_100k"][5]
    out = {}
    for shape in ("24", "12"):
        monkeypatch.setenv("UMAPB_KNN_SHAPE", shape)
        out[shape] = umap.knn(X, k)
    monkeypatch.delenv("UMAPB_KNN_SHAPE")
    assert np.array_equal(out["12"][0], out["24"][0]) and np.array_equal(out["12"][1], out["24"][1])
    rows = sampled_rows(X.shape[0], 4, 125, seed=9)
    ridx, rdist = oracle_knn_rows(X, k, rows, 125)
    assert same_neighbors(out["12"][0][rows], ridx, rdist) == 0
