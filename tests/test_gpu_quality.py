"""Layout quality on the benchmark workloads against the reference's own runs.

tests/golden/quality_<workload>.json holds the reference's fuzzy
cross-entropy and trustworthiness (k = 15, on a fixed sample of 10,000 query
points with the whole data set as candidates) for the benchmark's seeded data,
made by tests/golden/make_quality.py with the reference pipeline on the host
cores.  Here the device pipeline (initialize_from_data + run, same options) is
run on the same data and the same two measures are taken: trustworthiness
within 0.005 and cross-entropy within 1 % of the reference's mean over its
seeds.  The cross-entropy graph is built from the device's kNN after 500
sampled rows of it have been checked against the oracle's exact FP64 search.
"""
import glob
import json
import os

import numpy as np
import pytest

import bench
import oracle
from helpers import oracle_knn_rows, same_neighbors, sampled_rows, trustworthiness_torch

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "quality_*.json")))


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[8:-5] for p in FIXTURES])
def test_quality_matches_reference(umap, path):
    with open(path) as f:
        ref = json.load(f)
    n, k, epochs = ref["n"], ref["k"], ref["epochs"]
    X = bench.make_data(ref["workload"])
    assert X.shape == (n, ref["dim"])
    Y = np.zeros((n, 2), np.float32)
    st = umap.initialize_from_data(X, 2, Y, umap.Options(num_neighbors=k, num_epochs=epochs))
    st.run(Y)
    assert np.all(np.isfinite(Y))

    # the graph of the cross-entropy: FP64 similarities and union of the device's
    # exact kNN, checked first on sampled rows against the oracle's FP64 search
    idx, dist = umap.knn(X, k)
    rows = sampled_rows(n, 4, 125, seed=77)
    ridx, rdist = oracle_knn_rows(X, k, rows, 125)
    assert same_neighbors(idx[rows], ridx, rdist) == 0
    w, _, _ = oracle.neighbor_similarities(oracle.CSR.from_dense(idx, dist.astype(np.float64)))
    g = oracle.combine_neighbor_sets(w, 1.0)
    a, b = oracle.find_ab(1.0, 0.1)
    ce = oracle.cross_entropy(g, Y, a, b)
    q = np.sort(np.random.default_rng(ref["query_seed"]).choice(n, size=ref["num_queries"], replace=False))
    tr = trustworthiness_torch(X, Y, ref["trust_k"], queries=q)

    ce_ref = float(np.mean([r["cross_entropy"] for r in ref["reference"]]))
    tr_ref = float(np.mean([r["trustworthiness"] for r in ref["reference"]]))
    print(f"{ref['workload']}: trustworthiness {tr:.5f} (reference {tr_ref:.5f}, {tr - tr_ref:+.5f}); "
          f"cross-entropy {ce:.6g} (reference {ce_ref:.6g}, {100 * (ce - ce_ref) / ce_ref:+.3f} %)")
    assert abs(tr - tr_ref) <= 0.005, (tr, tr_ref)
    assert abs(ce - ce_ref) <= 0.01 * ce_ref, (ce, ce_ref)
