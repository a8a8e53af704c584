"""Reference layout quality on the 2000 x 10 N(0, 1) example (tests/golden/pipeline_quality_normal_2000.json).

The reference's serial optimize_layout (the oracle's restatement, bit-identical
to the reference headers compiled in oracle/_ref) from the spectral initial
layout, 500 epochs, for seeds 1234567890 + s, s = 0 .. SEEDS-1, in FP32 and
FP64.  Records each run's trustworthiness (k = 15) and fuzzy cross-entropy
over the union graph.  tests/test_gpu_pipeline.py compares the mean of the
device's runs on the same input with these means; tests/test_oracle.py
recomputes the first seed of each precision to pin the file to the oracle.

    python tests/golden/make_pipeline_quality.py [--seeds 48] [--workers 8]
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

N, DIM, K, EPOCHS, DATA_SEED, SEED_BASE = 2000, 10, 15, 500, 1000, 1234567890


def setup(dtype):
    """Data, union graph, epochs and spectral layout, as the device test builds them."""
    import oracle
    from helpers import neighbors_of, normal_data

    X = normal_data(N, DIM, seed=DATA_SEED, dtype=dtype)
    nl = neighbors_of(X, K)
    w64, _, _ = oracle.neighbor_similarities(nl.astype(np.float64))
    g = oracle.combine_neighbor_sets(oracle.CSR(nl.ptr, nl.idx, w64.val.astype(dtype)), 1.0)
    ep = oracle.similarities_to_epochs(g, EPOCHS, 5.0)
    ok, Y0, _ = oracle.spectral_init(g, 2)
    assert ok
    return X, g, ep, Y0


def reference_run(dtype, seed: int):
    """(trustworthiness, cross-entropy) of one reference run."""
    import oracle

    X, g, ep, Y0 = setup(dtype)
    a, b = oracle.find_ab(1.0, 0.1)
    R = Y0.copy()
    oracle.optimize_layout(2, R, ep.copy(), a, b, 1.0, 1.0, SEED_BASE + seed, EPOCHS)
    return float(oracle.trustworthiness(X, R, K)), float(oracle.cross_entropy(g.astype(np.float64), R, a, b))


def _job(args):
    name, seed = args
    return name, seed, reference_run(getattr(np, name), seed)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=48)
    ap.add_argument("--workers", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    jobs = [(name, s) for name in ("float32", "float64") for s in range(args.seeds)]
    with mp.get_context("spawn").Pool(args.workers) as pool:
        results = pool.map(_job, jobs)
    out = {"n": N, "dim": DIM, "k": K, "epochs": EPOCHS, "data_seed": DATA_SEED, "seed_base": SEED_BASE}
    for name in ("float32", "float64"):
        rows = sorted((s, r) for nm, s, r in results if nm == name)
        out[name] = {"seeds": [s for s, _ in rows], "trust": [r[0] for _, r in rows],
                     "cross_entropy": [r[1] for _, r in rows]}
        t = np.array(out[name]["trust"])
        print(name, "trust mean %.5f sd %.5f" % (t.mean(), t.std(ddof=1)))
    with open(os.path.join(HERE, "pipeline_quality_normal_2000.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
