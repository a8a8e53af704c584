"""Generates tests/golden/*.npz from the reference itself.

The outputs come from oracle/_ref/libumappp_ref.so: the reference's headers
(libscran/umappp v3.3.2, include/umappp/*.hpp) compiled unmodified against the
project's stand-ins for its absent dependencies (oracle/ref_shim).  The
fixtures pin the C restatement in oracle/ on machines without the reference
sources.  Run from the repository root:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402


def case(name: str, n: int, dim: int, k: int, dtype, seed: int, num_epochs: int = 100):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, dim)).astype(dtype)
    idx, dist = oracle.ref_knn(X, k)
    nl = oracle.CSR.from_dense(idx, dist)
    sims = oracle.ref_neighbor_similarities(nl)
    sims_conn = oracle.ref_neighbor_similarities(nl, local_connectivity=1.3, use_newton=False)
    union = oracle.ref_combine_neighbor_sets(sims, 1.0)
    inter = oracle.ref_combine_neighbor_sets(sims, 0.0)
    mixed = oracle.ref_combine_neighbor_sets(sims, 0.5)
    ep = oracle.ref_similarities_to_epochs(union, num_epochs, 5.0)
    ok, Y0 = oracle.ref_spectral_init(union, 2)
    Y = Y0.copy()
    ep_run = ep.copy()
    a, b = oracle.ref_find_ab(1.0, 0.1)
    oracle.ref_optimize_layout(2, Y, ep_run, a, b, 1.0, 1.0, 1234567890, num_epochs)
    rnd = oracle.ref_random_init(n, 2, seed=seed, dtype=dtype)
    out = dict(
        X=X, knn_idx=idx, knn_dist=dist, sims=sims.val, sims_conn13_bisect=sims_conn.val,
        union_ptr=union.ptr, union_idx=union.idx, union_val=union.val,
        inter_ptr=inter.ptr, inter_idx=inter.idx, inter_val=inter.val,
        mixed_ptr=mixed.ptr, mixed_idx=mixed.idx, mixed_val=mixed.val,
        ep_ptr=ep.ptr, ep_targets=ep.targets, ep_eps=ep.eps, ep_enext=ep.enext, ep_enneg=ep.enneg,
        spectral_ok=np.array(ok), spectral_Y=Y0, sgd_Y=Y, sgd_enext=ep_run.enext, sgd_enneg=ep_run.enneg,
        random_init=rnd, num_epochs=np.array(num_epochs), ab=np.array([a, b]),
    )
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


def scalars():
    ab = {f"{s}_{m}": oracle.ref_find_ab(s, m) for s, m in ((1, 0.05), (1, 0.01), (2, 0.1), (200, 1), (20, 1000), (1, 0.1))}
    epochs = {str(n): oracle.ref().ref_choose_num_epochs(0, 0, n) for n in (1000, 10000, 10001, 20000, 10000000)}
    np.savez_compressed(os.path.join(HERE, "scalars.npz"),
                        ab_keys=np.array(list(ab.keys())), ab_vals=np.array(list(ab.values())),
                        epoch_n=np.array([int(x) for x in epochs]), epoch_vals=np.array(list(epochs.values())))


if __name__ == "__main__":
    oracle.build()
    case("small_f64", 200, 5, 15, np.float64, seed=1)
    case("small_f32", 150, 7, 10, np.float32, seed=2)
    scalars()
    print("written to", HERE)
