"""Reference layout quality on the benchmark workloads (tests/golden/quality_<workload>.json).

Runs the reference pipeline (oracle/_ref/libumappp_ref.so: the reference's
headers compiled against the project's stand-ins) on the host cores, on the
benchmark's seeded Gaussian mixture: exact kNN (the reference's brute-force
search), initialize() and Status::run() with the benchmark's options, for a
few optimisation seeds.  Records, per seed, the fuzzy cross-entropy of the
layout over the union graph and its trustworthiness (k = 15) on a fixed,
seeded sample of 10,000 query points (the full data set as candidates).  The device test
(tests/test_gpu_quality.py) recomputes both for the device's layout on the
same data and queries.

    python tests/golden/make_quality.py [--workload mixture_1m] [--seeds 2]
        [--knn-cache PATH]     # .npz with the kNN, reused if present
        [--layouts-out DIR | --layouts-in DIR] [--only cross_entropy|trustworthiness]
        [--out PATH]

The 1M-point workload takes about half an hour on 8 cores for the exact kNN
and seven minutes per seed for the reference's SGD.  Its 10,000-query
trustworthiness takes hours on host cores but seconds on a GPU, so the two
halves can run apart: --layouts-out writes the reference's layouts (raw
float32) and stops; --layouts-in reads them and takes the measures (with
torch on a GPU when one is present).  --only takes one of the two measures
and merges it into an existing fixture for the same workload and seeds, so the
cross-entropy (which needs the kNN graph) can be taken where the kNN is, and
the trustworthiness (which needs only the data and the layouts) on a GPU.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
import oracle  # noqa: E402

sys.path.insert(0, os.path.dirname(HERE))
from helpers import trustworthiness_torch  # noqa: E402

QUERY_SEED = 123
NUM_QUERIES = 10000


def query_sample(n: int) -> np.ndarray:
    return np.sort(np.random.default_rng(QUERY_SEED).choice(n, size=min(NUM_QUERIES, n), replace=False)).astype(np.int32)


def measures(X, g, a, b, Y, q, only=None):
    """Cross-entropy over the union graph (oracle, FP64) and trustworthiness on
    the query sample (tests/helpers.trustworthiness_torch, equal to
    oracle.trustworthiness; on a GPU when there is one).  With 'only', the
    other measure is None."""
    import torch

    device = "cuda" if torch.cuda.is_available() else "cpu"
    ce = oracle.cross_entropy(g, Y, a, b) if only in (None, "cross_entropy") else None
    tr = trustworthiness_torch(X, Y, 15, queries=q, device=device, batch=16 if device == "cpu" else 8) \
        if only in (None, "trustworthiness") else None
    return ce, tr


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="mixture_1m", choices=sorted(bench.CONFIGS))
    ap.add_argument("--seeds", type=int, default=2)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--knn-cache", default=None)
    ap.add_argument("--layouts-out", default=None,
                    help="write the reference layouts (<dir>/<workload>_<seed>.f32) and stop before the measures")
    ap.add_argument("--layouts-in", default=None, help="take the reference layouts from this directory")
    ap.add_argument("--only", default=None, choices=["cross_entropy", "trustworthiness"],
                    help="take one measure and merge it into the existing fixture")
    ap.add_argument("--out", default=None, help="fixture path (default tests/golden/quality_<workload>.json)")
    args = ap.parse_args()

    n, dim, _, _, _, k, epochs = bench.CONFIGS[args.workload]
    X = bench.make_data(args.workload)
    if args.only is not None and not args.layouts_in:
        ap.error("--only measures the layouts of --layouts-in")
    nl = g = None
    a, b = oracle.find_ab(1.0, 0.1)
    if args.only != "trustworthiness":   # the trustworthiness alone needs no kNN
        t0 = time.time()
        if args.knn_cache and os.path.exists(args.knn_cache):
            z = np.load(args.knn_cache)
            idx, dist = z["idx"], z["dist"]
        else:
            idx, dist = oracle.ref_knn(X, k, nthreads=args.threads)
            if args.knn_cache:
                np.savez(args.knn_cache, idx=idx, dist=dist)
        print(f"knn {time.time() - t0:.0f} s", flush=True)
        nl = oracle.CSR.from_dense(idx, dist)
        w, _, _ = oracle.neighbor_similarities(nl.astype(np.float64))
        g = oracle.combine_neighbor_sets(w, 1.0)
    q = query_sample(n)

    runs = []
    for s in range(args.seeds):
        seed = 1234567890 + s
        path = lambda d: os.path.join(d, f"{args.workload}_{seed}.f32")  # noqa: E731
        secs = None
        if args.layouts_in:
            Y = np.fromfile(path(args.layouts_in), dtype=np.float32).reshape(n, 2)
        else:
            Y = np.zeros((n, 2), np.float32)
            t0 = time.time()
            st = oracle.ref_initialize(nl, 2, Y, num_epochs=epochs, optimize_seed=seed, num_threads=args.threads,
                                       num_threads_optimize=args.threads, num_threads_spectral=args.threads)
            st.run(Y)
            secs = round(time.time() - t0, 1)
        if args.layouts_out:
            os.makedirs(args.layouts_out, exist_ok=True)
            Y.tofile(path(args.layouts_out))
            print("wrote", path(args.layouts_out), secs, flush=True)
            continue
        ce, tr = measures(X, g, a, b, Y, q, args.only)
        run = {"optimize_seed": seed, "cross_entropy": ce, "trustworthiness": tr, "seconds": secs}
        runs.append({key: v for key, v in run.items() if v is not None or key == "seconds"})
        print(runs[-1], flush=True)
    if args.layouts_out:
        return

    out = {
        "workload": args.workload, "n": n, "dim": dim, "k": k, "epochs": epochs,
        "data": "bench.make_data(workload) (seeded Gaussian mixture)",
        "trust_k": 15, "query_seed": QUERY_SEED, "num_queries": int(len(q)),
        "cross_entropy_graph": "FP64 similarities + union of the exact kNN, oracle.cross_entropy",
        "reference": runs,
    }
    path = args.out or os.path.join(HERE, f"quality_{args.workload}.json")
    if args.only is not None and os.path.exists(path):
        with open(path) as f:
            old = json.load(f)
        same = (old.get("workload") == args.workload and old.get("query_seed") == QUERY_SEED
                and old.get("num_queries") == len(q))
        by_seed = {r["optimize_seed"]: r for r in old["reference"]} if same else {}
        for r in runs:   # keep the other measure (and the timing) of the same seed
            merged = dict(by_seed.get(r["optimize_seed"], {}))
            merged.update({key: v for key, v in r.items() if v is not None})
            r.clear()
            r.update(merged)
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
