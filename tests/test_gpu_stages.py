"""Parity of each device stage with the oracle, through the C ABI.

Tolerances (stated per test): integer, index and graph-structure outputs are
bit-exact; FP64 values within 1e-12 relative; FP32-stored values computed in
FP64 within 1e-6 relative (the bar for weights and rho/sigma).
"""
import numpy as np
import pytest

import oracle
from helpers import (csr_tuple, eigen_check, mock_probabilities, neighbors_of, normal_data, rel_err,
                     same_neighbors, two_populations)

pytestmark = pytest.mark.gpu


# ------------------------------------------------------------------ kNN ---

# (12, 4, 5), (20, 3, 10): fewer other points than the candidate list holds, so
# padding columns of the tensor-core tile must never become candidates
@pytest.mark.parametrize("n,dim,k", [(2000, 10, 15), (1500, 50, 15), (600, 7, 5), (300, 3, 30), (12, 4, 5),
                                     (20, 3, 10), (129, 6, 15)])
def test_knn_f32_matches_fp64_bruteforce(umap, n, dim, k):
    X = oracle.gaussian_mixture(n, dim, 6, 4.0, seed=n + dim, dtype=np.float32)
    idx, dist = umap.knn(X, k)
    ridx, rdist = oracle.knn(X, k)
    assert same_neighbors(idx, ridx, rdist) == 0
    # distances are FP64 results rounded to float
    assert rel_err(dist, rdist) <= 1e-6


@pytest.mark.parametrize("n,dim,k", [(2000, 10, 15), (500, 5, 10)])
def test_knn_f64_bit_exact(umap, n, dim, k):
    X = normal_data(n, dim, seed=7 * n)
    idx, dist = umap.knn(X, k)
    ridx, rdist = oracle.knn(X, k)
    assert np.array_equal(idx, ridx)
    assert np.array_equal(dist, rdist)


@pytest.mark.parametrize("kind", ["f16", "tf32"])
@pytest.mark.parametrize("n,dim,k", [(3000, 50, 15), (2500, 90, 10), (700, 20, 20), (300, 63, 15)])
def test_knn_tensor_core_operands(umap, monkeypatch, kind, n, dim, k):
    # both operand splits give the exact neighbours; the candidate distances stay
    # inside the bound that decides FP64 recomputation (2^-17 of |q|^2 + max |r|^2)
    monkeypatch.setenv("UMAPB_KNN_TC_KIND", kind)
    X = oracle.gaussian_mixture(n, dim, 8, 3.0, seed=n + dim + k, dtype=np.float32)
    X *= np.float32(37.5)   # not a power of two: the FP16 scaling must stay exact
    idx, dist = umap.knn(X, k)
    ridx, rdist = oracle.knn(X, k)
    assert same_neighbors(idx, ridx, rdist) == 0
    assert rel_err(dist, rdist) <= 1e-6
    err = umap.lib().umapb_knn_last_tc_error()
    if kind == "tf32" and dim + 1 > 64:
        assert err == 0.0          # no TF32 tensor-core path at this width: SIMT search
    else:
        assert 0.0 < err < 2.0 ** -17, err


@pytest.mark.parametrize("prune", ["1", "0"])
def test_knn_tile_pruning_is_exact(umap, monkeypatch, prune):
    # well separated clusters: most reference tiles are provably too far for a
    # query block and are skipped; the neighbours stay exact
    monkeypatch.setenv("UMAPB_KNN_PRUNE", prune)
    n = 20000
    X = oracle.gaussian_mixture(n, 30, 8, 10.0, seed=11, dtype=np.float32)
    idx, dist = umap.knn(X, 15)
    ridx, rdist = oracle.knn(X, 15)
    assert same_neighbors(idx, ridx, rdist) == 0
    assert rel_err(dist, rdist) <= 1e-6
    pairs = umap.lib().umapb_knn_last_tile_pairs()
    tiles = (n + 127) // 128
    if prune == "1":
        assert 0 < pairs < 0.5 * tiles * tiles, pairs
    else:
        assert pairs >= tiles * tiles, pairs


def test_knn_duplicates_and_ties(umap):
    rng = np.random.default_rng(3)
    base = rng.normal(size=(50, 4))
    X = np.concatenate([base, base, base[:10]]).astype(np.float32)   # exact duplicates: distance 0 ties
    idx, dist = umap.knn(X, 6)
    ridx, rdist = oracle.knn(X, 6)
    assert np.array_equal(dist.astype(np.float64) == 0, rdist == 0)
    assert same_neighbors(idx, ridx, rdist) == 0


def test_knn_rejects_bad_k(umap):
    X = np.zeros((5, 2), np.float32)
    with pytest.raises(umap.UmapbError):
        umap.knn(X, 5)


# --------------------------------------------------------- similarities ---

@pytest.mark.parametrize("n", [50, 200])
@pytest.mark.parametrize("k", [5, 10, 20])
@pytest.mark.parametrize("conn", [0.4, 1.0, 1.3, 2.0, 2.5])
@pytest.mark.parametrize("newton", [True, False])
def test_similarities_f64(umap, n, k, conn, newton):
    nl = neighbors_of(normal_data(n, 5, seed=int(n * k + conn * 10)), k)
    (_, _, w), rho, sigma = umap.neighbor_similarities(csr_tuple(nl), local_connectivity=conn, use_newton=newton,
                                                       return_rho_sigma=True)
    rw, rrho, rsig = oracle.neighbor_similarities(nl, local_connectivity=conn, use_newton=newton)
    assert rel_err(w, rw.val) <= 1e-12
    ok = ~np.isnan(rrho)
    assert np.array_equal(np.isnan(rho), np.isnan(rrho))
    assert rel_err(rho[ok], rrho[ok]) <= 1e-12
    ok = ~np.isnan(rsig)
    assert rel_err(sigma[ok], rsig[ok]) <= 1e-12
    # the reference's own checks (tests/src/neighbor_similarities.cpp:52-80), with the sigma floor off
    (_, _, w2) = umap.neighbor_similarities(csr_tuple(nl), local_connectivity=conn, use_newton=newton,
                                            min_k_dist_scale=1e-8)
    for i in range(n):
        row = w2[nl.ptr[i]:nl.ptr[i + 1]]
        assert np.all(row[: int(conn)] == 1)
        assert np.all(row[int(conn):] < 1)
        assert np.all(np.diff(row) <= 0)
        assert abs(row.sum() - np.log2(len(row) + 1)) < 1e-5


@pytest.mark.parametrize("conn", [0.4, 1.0, 2.5])
def test_similarities_f32_against_fp64_oracle(umap, conn):
    nl = neighbors_of(normal_data(300, 8, seed=11), 15, dtype=np.float32)
    (_, _, w), rho, sigma = umap.neighbor_similarities(csr_tuple(nl), local_connectivity=conn, return_rho_sigma=True)
    rw, rrho, rsig = oracle.neighbor_similarities(nl.astype(np.float64), local_connectivity=conn)
    assert w.dtype == np.float32
    assert rel_err(w, rw.val) <= 1e-6
    assert rel_err(rho, rrho) <= 1e-6
    assert rel_err(sigma, rsig) <= 1e-6
    # against the reference's float arithmetic: same search, float rounding only
    fw, _, _ = oracle.neighbor_similarities(nl, local_connectivity=conn)
    assert rel_err(w, fw.val) <= 1e-4


def test_similarities_edge_cases(umap):
    # empty row, all-zero distances, all ties, connectivity too high (neighbor_similarities.cpp:130-190)
    rows = [[], [(j, 0.0) for j in range(1, 21)], [(j, 10.0) for j in range(20)],
            [(j, j * 0.1) for j in range(20)]]
    ptr, idx, val = umap.to_csr(rows)
    _, _, w = umap.neighbor_similarities((ptr, idx, val))
    assert np.all(w[ptr[1]:ptr[4]][:40] == 1)
    _, _, w = umap.neighbor_similarities((ptr, idx, val), local_connectivity=100.0)
    assert np.all(w == 1)


def test_similarities_bounded_sigma(umap):
    # neighbor_similarities.cpp:192-228: bandwidth 0 drives sigma down until the floor
    rows = [[(j, j * 0.1 + 0.01) for j in range(20)] for _ in range(3)]
    ptr, idx, val = umap.to_csr(rows, np.float32)
    _, _, w = umap.neighbor_similarities((ptr, idx, val), bandwidth=0.0, min_k_dist_scale=0.1, use_newton=False)
    assert np.all(w <= 1) and np.all(w > 0)
    _, _, w0 = umap.neighbor_similarities((ptr, idx, val), bandwidth=0.0, min_k_dist_scale=0.0, use_newton=False)
    w0 = w0.reshape(3, 20)
    assert np.all(w0[:, 0] == 1) and np.all(w0[:, 1:] == 0)
    rw, _, _ = oracle.neighbor_similarities(oracle.CSR(ptr, idx, val.astype(np.float64)), bandwidth=0.0,
                                            min_k_dist_scale=0.1, use_newton=False)
    assert rel_err(w, rw.val) <= 1e-6


# ----------------------------------------------------------------- union ---

@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n,k", [(50, 5), (100, 10), (200, 15), (3000, 15)])
@pytest.mark.parametrize("mix", [1.0, 0.0, 0.5])
def test_union_bit_exact(umap, dtype, n, k, mix):
    nl = neighbors_of(normal_data(n, 5, seed=n * k), k, dtype=dtype)
    nl.val = np.exp(-nl.val).astype(dtype)          # combine_neighbor_sets.cpp:36-41
    ptr, idx, val = umap.combine_neighbor_sets(csr_tuple(nl), mix)
    ref = oracle.combine_neighbor_sets(nl, mix)
    assert np.array_equal(ptr, ref.ptr)
    assert np.array_equal(idx, ref.idx)
    assert np.array_equal(val, ref.val)


def test_union_rejects_bad_neighbors(umap):
    rows = [[(0, 0.5)], [(0, 0.5)]]    # self edge in row 0
    with pytest.raises(umap.UmapbError):
        umap.combine_neighbor_sets(rows)


# ---------------------------------------------------------------- epochs ---

@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n,k", [(50, 5), (200, 15), (3000, 15)])
def test_epochs_bit_exact(umap, dtype, n, k):
    nl = neighbors_of(normal_data(n, 5, seed=n + k), k, dtype=dtype)
    w, _, _ = oracle.neighbor_similarities(nl)
    g = oracle.combine_neighbor_sets(w, 1.0)
    g.val[0] = dtype(1e-8)                     # optimize_layout.cpp:58-77: this edge must be removed
    ep = umap.similarities_to_epochs(csr_tuple(g), 500, 5.0)
    ref = oracle.similarities_to_epochs(g, 500, 5.0)
    assert np.array_equal(ep.cumulative_num_edges, ref.ptr)
    assert np.array_equal(ep.edge_targets, ref.targets)
    for a, b in ((ep.epochs_per_sample, ref.eps), (ep.epoch_of_next_sample, ref.enext),
                 (ep.epoch_of_next_negative_sample, ref.enneg)):
        assert np.array_equal(a, b)
    assert len(ep.edge_targets) < g.nnz
    assert np.all(ep.epochs_per_sample >= 1)


# ------------------------------------------------------------ components ---

def _symmetrize(rows):
    out = [list(r) for r in rows]
    for i, r in enumerate(rows):
        for j, v in r:
            out[j].append((i, v))
    return [sorted(r) for r in out]


def test_components_hand_cases(umap):
    # tests/src/spectral_init.cpp:176-224
    e = [[] for _ in range(5)]
    e[4] += [(0, 0.5), (1, 0.5)]
    e[3] += [(2, 0.5)]
    assert umap.has_multiple_components(_symmetrize(e))
    e[3] += [(1, 0.5)]
    assert not umap.has_multiple_components(_symmetrize(e))
    assert umap.has_multiple_components([[] for _ in range(5)])
    e = [[] for _ in range(6)]
    e[4] += [(2, 0.5), (3, 0.5)]
    e[5] += [(1, 0.5), (0, 0.5)]
    assert umap.has_multiple_components(_symmetrize(e))


@pytest.mark.parametrize("n", [50, 500])
def test_components_random(umap, n):
    g = mock_probabilities(n, seed=n)
    assert not umap.has_multiple_components(csr_tuple(g))
    two = oracle.CSR.from_lists(g.to_lists() + [[(j + n, v) for j, v in r] for r in g.to_lists()])
    assert umap.has_multiple_components(csr_tuple(two)) == oracle.has_multiple_components(two) == True


# -------------------------------------------------------------- spectral ---

@pytest.mark.parametrize("n", [50, 100, 200])
@pytest.mark.parametrize("ndim", [2, 5])
def test_spectral_init(umap, n, ndim):
    g = mock_probabilities(n, seed=n)
    irl = umap.IrlbaOptions(convergence_tolerance=1e-8) if hasattr(umap, "IrlbaOptions") else None
    ok, Y, ev = umap.spectral_init(csr_tuple(g), ndim, irlba=irl, return_evals=True)
    rok, rY, rev = oracle.spectral_init(g, ndim, tol=1e-8)
    assert ok and rok
    assert np.all(Y != 0)
    assert abs(np.abs(Y).max() - 10) < 1e-12
    assert eigen_check(g, Y)
    assert rel_err(ev, rev) <= 1e-9
    # same vectors as the FP64 oracle up to sign, where the eigenvalues are separated
    for d in range(ndim):
        gap = min(abs(rev[d + 1] - rev[d]), abs(rev[d + 1] - rev[d + 2]) if d + 2 < len(rev) else 1.0)
        if gap > 1e-3:
            s = np.sign(np.dot(Y[:, d], rY[:, d]))
            assert np.max(np.abs(Y[:, d] - s * rY[:, d])) < 1e-5


def test_spectral_multi_component_fails(umap):
    g = mock_probabilities(50, seed=1)
    g2 = mock_probabilities(100, seed=2)
    two = oracle.CSR.from_lists(g.to_lists() + [[(j + 50, v) for j, v in r] for r in g2.to_lists()])
    ok, Y = umap.spectral_init(csr_tuple(two), 2)
    assert not ok
    assert np.all(Y == 0)


def test_spectral_jitter_changes_output(umap):
    g = mock_probabilities(51, seed=51)
    ok, Y = umap.spectral_init(csr_tuple(g), 3)
    ok2, Yj = umap.spectral_init(csr_tuple(g), 3, jitter=True, jitter_sd=1e-3, seed=69)
    assert ok and ok2
    assert not np.array_equal(Y, Yj)
    assert Y.reshape(-1)[-1] != Yj.reshape(-1)[-1]
    assert np.max(np.abs(Y - Yj)) < 0.01


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_random_init_range(umap, dtype):
    Y = umap.random_init(1000, 3, seed=69, scale=10, dtype=dtype)
    assert np.all(Y != 0) and np.all(Y >= -10) and np.all(Y < 10)
    assert abs(Y.mean()) < 0.5 and 5.0 < Y.std() < 6.5


# --------------------------------------------------------------- schedule ---

@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_schedule_counts_exact(umap, dtype):
    nl = neighbors_of(two_populations(400, 5, seed=4), 15, dtype=dtype)
    # the oracle's union and schedule from the device's own weights
    _, _, wd = umap.neighbor_similarities(csr_tuple(nl))
    w = oracle.CSR(nl.ptr, nl.idx, wd)
    g = oracle.combine_neighbor_sets(w, 1.0)
    Y = np.ascontiguousarray(oracle.random_init(400, 2, dtype=dtype))
    st = umap.initialize(csr_tuple(nl), 2, Y.copy(), umap.Options(initialize_method=umap.InitializeMethod.NONE,
                                                                  num_epochs=300))
    counts = st.schedule_counts()
    ep = oracle.similarities_to_epochs(g, 300, 5.0)
    ref = oracle.optimize_layout(2, Y.copy(), ep, 1.577, 0.895, 1.0, 1.0, 1234567890, 300, counts=True)
    assert np.array_equal(counts, ref)


# ---------------------------------------------------------------- adjoint ---

@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_loss_grad_matches_oracle(umap, dtype):
    nl = neighbors_of(normal_data(300, 6, seed=5), 10)
    w, _, _ = oracle.neighbor_similarities(nl)
    g = oracle.combine_neighbor_sets(w, 1.0)
    Y = np.random.default_rng(1).normal(size=(300, 2)) * 3
    a, b = oracle.find_ab(1.0, 0.1)
    loss, gY, gab = umap.loss_grad(csr_tuple(g.astype(dtype)), Y.astype(dtype), a, b)
    rl, rgY, rgab = oracle.loss_grad(g.astype(dtype).astype(np.float64), Y.astype(dtype).astype(np.float64), a, b)
    tol = 1e-10 if dtype == np.float64 else 1e-6
    assert abs(loss - rl) <= tol * abs(rl)
    assert np.max(np.abs(gY - rgY)) <= tol * np.max(np.abs(rgY))
    assert np.max(np.abs(np.array(gab) - rgab)) <= 1e-9 * np.max(np.abs(rgab))


def test_loss_grad_rejects_out_of_range_indices(umap):
    """A neighbour index outside [0, num_obs) is skipped on the device and
    reported as an invalid argument instead of being read."""
    nl = neighbors_of(normal_data(200, 6, seed=6), 10)
    w, _, _ = oracle.neighbor_similarities(nl)
    g = oracle.combine_neighbor_sets(w, 1.0)
    Y = np.random.default_rng(2).normal(size=(200, 2))
    a, b = oracle.find_ab(1.0, 0.1)
    idx = g.idx.copy()
    idx[3] = 200
    with pytest.raises(umap.UmapbError, match="out of range"):
        umap.loss_grad((g.ptr, idx, g.val), Y, a, b)
    loss, _, _ = umap.loss_grad(csr_tuple(g), Y, a, b)   # the next call is unaffected
    assert np.isfinite(loss)
