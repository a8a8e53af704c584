"""End-to-end parity of initialize() / Status::run() with the reference.

The reference path is the oracle's serial optimize_layout (bit-identical to
the reference headers compiled in oracle/_ref) from the same initial layout.
Parallel SGD reorders updates and draws its negative samples from a
different generator, so layouts are compared by quality:
trustworthiness(k=15) within 0.005 and fuzzy cross-entropy within 1%.
Everything RNG-free is compared exactly.
"""
import json
import os

import numpy as np
import pytest

import oracle
from helpers import csr_tuple, mock_neighbors, neighbors_of, normal_data, rel_err, two_populations

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _oracle_pipeline(nl: oracle.CSR, dtype, num_epochs, rate=5.0, device_weights=None):
    """Similarities (FP64, stored in dtype) -> union -> epochs, as the device computes them.
    With device_weights, the oracle's union and schedule start from the device's weights."""
    if device_weights is None:
        w64, _, _ = oracle.neighbor_similarities(nl.astype(np.float64))
        w = oracle.CSR(nl.ptr, nl.idx, w64.val.astype(dtype))
    else:
        w = oracle.CSR(nl.ptr, nl.idx, np.asarray(device_weights, dtype=dtype))
    g = oracle.combine_neighbor_sets(w, 1.0)
    return g, oracle.similarities_to_epochs(g, num_epochs, rate)


def _device_weights(umap, nl):
    _, _, w = umap.neighbor_similarities(csr_tuple(nl))
    return w


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_epoch_data_matches_oracle(umap, dtype):
    nl = neighbors_of(normal_data(500, 10, seed=2), 15, dtype=dtype)
    Y = np.zeros((500, 2), dtype=dtype)
    st = umap.initialize(csr_tuple(nl), 2, Y, umap.Options(initialize_method=umap.InitializeMethod.NONE))
    assert st.epoch() == 0 and st.num_epochs() == 500 and st.num_observations() == 500
    a, b = oracle.find_ab(1.0, 0.1)
    assert (st.a, st.b) == (a, b)
    ep = st.get_epoch_data()
    # from the device's weights, the union and the schedule are bit-exact
    _, ref = _oracle_pipeline(nl, dtype, 500, device_weights=_device_weights(umap, nl))
    assert np.array_equal(ep.cumulative_num_edges, ref.ptr)
    assert np.array_equal(ep.edge_targets, ref.targets)
    assert np.array_equal(ep.epochs_per_sample, ref.eps)
    assert np.array_equal(ep.epoch_of_next_sample, ref.enext)
    assert np.array_equal(ep.epoch_of_next_negative_sample, ref.enneg)
    # against the host's weights: the device exp is correctly rounded, the host
    # libm's exp is not always, so single weights may differ in the last bit
    _, ref2 = _oracle_pipeline(nl, dtype, 500)
    assert np.array_equal(ep.edge_targets, ref2.targets)
    tol = 1e-12 if dtype == np.float64 else 1e-6
    assert rel_err(ep.epochs_per_sample, ref2.eps) <= tol
    assert np.mean(ep.epochs_per_sample == ref2.eps) > 0.95


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_layout_quality_matches_reference(umap, dtype):
    n = 2000
    X = normal_data(n, 10, seed=1000, dtype=dtype)        # the README's 2000 x 10 N(0,1) example shape
    nl = neighbors_of(X, 15)
    g, _ = _oracle_pipeline(nl, dtype, 500)
    ok, Y0, _ = oracle.spectral_init(g, 2)
    assert ok
    # At 2000 points a single run's trustworthiness varies by about 0.0045 and its
    # cross-entropy by about 1% from seed to seed (in the reference too), as much
    # as the bars themselves.  So the mean over 16 device runs (different optimize
    # seeds) is compared with the mean over the reference's runs in
    # tests/golden/pipeline_quality_normal_2000.json (its serial SGD from the same
    # initial layout, 48 seeds; made by tests/golden/make_pipeline_quality.py):
    # within 0.005 / 1%, or within 2.5 standard errors of the difference of the
    # means where that is larger.
    with open(os.path.join(GOLDEN, "pipeline_quality_normal_2000.json")) as f:
        ref = json.load(f)
    assert (ref["n"], ref["dim"], ref["k"], ref["epochs"], ref["data_seed"]) == (n, 10, 15, 500, 1000)
    t_ref = np.array(ref[np.dtype(dtype).name]["trust"])
    ce_ref = np.array(ref[np.dtype(dtype).name]["cross_entropy"])
    a, b = oracle.find_ab(1.0, 0.1)
    gw = g.astype(np.float64)
    t_dev, ce_dev = [], []
    for seed in range(16):
        Y = np.ascontiguousarray(Y0.copy())
        st = umap.initialize(csr_tuple(nl), 2, Y, umap.Options(initialize_method=umap.InitializeMethod.NONE,
                                                                optimize_seed=1234567890 + 101 * seed))
        st.run(Y)
        assert st.epoch() == 500
        assert np.all(np.isfinite(Y))
        t_dev.append(oracle.trustworthiness(X, Y, 15))
        ce_dev.append(oracle.cross_entropy(gw, Y, a, b))

    def se(x, y):
        return float(np.sqrt(np.var(x, ddof=1) / len(x) + np.var(y, ddof=1) / len(y)))

    t_bar = max(0.005, 2.5 * se(t_dev, t_ref))
    ce_bar = max(0.01 * np.mean(ce_ref), 2.5 * se(ce_dev, ce_ref))
    assert abs(np.mean(t_dev) - np.mean(t_ref)) <= t_bar, (np.mean(t_dev), np.mean(t_ref), t_dev)
    assert abs(np.mean(ce_dev) - np.mean(ce_ref)) <= ce_bar, (np.mean(ce_dev), np.mean(ce_ref), ce_dev)


def test_spectral_initialize_matches_reference(umap):
    X = normal_data(2000, 10, seed=1000)
    nl = neighbors_of(X, 15)
    Y = np.zeros((2000, 2))
    st = umap.initialize(csr_tuple(nl), 2, Y)
    g, _ = _oracle_pipeline(nl, np.float64, 500)
    ok, R, _ = oracle.spectral_init(g, 2)
    assert ok
    for d in range(2):
        s = np.sign(np.dot(Y[:, d], R[:, d]))
        assert np.max(np.abs(Y[:, d] - s * R[:, d])) < 1e-3 * 10


@pytest.mark.parametrize("n,k", [(50, 5), (100, 10), (200, 15)])
def test_two_populations_separate(umap, n, k):
    # tests/src/umappp.cpp:60-90
    X = two_populations(n, 5, seed=n * k)
    nl = neighbors_of(X, k)
    Y = np.zeros((n, 2))
    st = umap.initialize(csr_tuple(nl), 2, Y)
    assert st.num_epochs() == 500
    st.run(Y)
    assert st.epoch() == 500 and np.all(np.isfinite(Y))
    even, odd = Y[0::2], Y[1::2]
    sep = any(even[:, d].max() < odd[:, d].min() or odd[:, d].max() < even[:, d].min() for d in range(2))
    assert sep


def test_builder_path_equals_neighbor_path(umap):
    X = two_populations(300, 5, seed=9, dtype=np.float32)
    Y1 = np.zeros((300, 2), np.float32)
    s1 = umap.initialize_from_data(X, 2, Y1, umap.Options(num_neighbors=10))
    idx, dist = umap.knn(X, 10)
    Y2 = np.zeros((300, 2), np.float32)
    s2 = umap.initialize((idx, dist), 2, Y2, umap.Options())
    assert np.array_equal(Y1, Y2)
    e1, e2 = s1.get_epoch_data(), s2.get_epoch_data()
    assert np.array_equal(e1.edge_targets, e2.edge_targets)
    assert np.array_equal(e1.epochs_per_sample, e2.epochs_per_sample)


def test_partial_runs_follow_the_same_schedule(umap):
    # tests/src/umappp.cpp:104-115: run(200) then run() covers the same epochs as run()
    X = two_populations(200, 5, seed=5)
    nl = neighbors_of(X, 15)
    Y = np.zeros((200, 2))
    st = umap.initialize(csr_tuple(nl), 2, Y)
    Y0 = Y.copy()
    st.run(Y, 200)
    assert st.epoch() == 200
    assert not np.array_equal(Y, Y0)
    mid = st.get_epoch_data()
    st.run(Y)
    assert st.epoch() == 500
    full = umap.initialize(csr_tuple(nl), 2, np.zeros((200, 2)))
    assert np.array_equal(full.schedule_counts(200, 500), st.schedule_counts(200, 500))
    # the schedule state after 200 epochs is the reference's (from the same weights)
    _, ep = _oracle_pipeline(nl, np.float64, 500, device_weights=_device_weights(umap, nl))
    R = Y0.copy()
    oracle.optimize_layout(2, R, ep, st.a, st.b, 1.0, 1.0, 1, 200)
    assert np.array_equal(mid.epoch_of_next_sample, ep.enext)
    assert np.array_equal(mid.epoch_of_next_negative_sample, ep.enneg)


@pytest.mark.parametrize("n,epochs", [(3000, 500), (20000, 200)])
def test_event_windows_self_check(umap, monkeypatch, n, epochs):
    # every window's event lists are checked on the device against the
    # schedule recomputed from the initial state (counts, negatives, head order),
    # and its head segments (in order, one head each, at most the cap long)
    monkeypatch.setenv("UMAPB_CHECK_SCHEDULE", "1")
    X = oracle.gaussian_mixture(n, 12, 5, 4.0, seed=n, dtype=np.float32)
    Y = np.zeros((n, 2), np.float32)
    st = umap.initialize_from_data(X, 2, Y, umap.Options(num_epochs=epochs))
    st.run(Y, epochs // 3)
    st.run(Y)
    assert st.epoch() == epochs and np.all(np.isfinite(Y))


def test_many_small_windows(umap, monkeypatch):
    # window buffers capped at 2 MiB: about four epochs per window at 3000
    # points, so the two buffers alternate dozens of times (each window built
    # while the previous one's epochs run) and partial runs pick up a window
    # left by the last call; every window is checked on the device against the
    # recomputed schedule
    monkeypatch.setenv("UMAPB_SGD_WINDOW_BYTES", str(2 << 20))
    monkeypatch.setenv("UMAPB_CHECK_SCHEDULE", "1")
    n, epochs = 3000, 300
    X = oracle.gaussian_mixture(n, 12, 5, 4.0, seed=77, dtype=np.float32)
    Y = np.zeros((n, 2), np.float32)
    st = umap.initialize_from_data(X, 2, Y, umap.Options(num_epochs=epochs))
    for limit in (1, 37, 150, epochs):
        st.run(Y, limit)
        assert st.epoch() == limit
    assert np.all(np.isfinite(Y))
    monkeypatch.delenv("UMAPB_SGD_WINDOW_BYTES")
    Z = np.zeros((n, 2), np.float32)
    one = umap.initialize_from_data(X, 2, Z, umap.Options(num_epochs=epochs))
    one.run(Z)
    t_many, t_one = oracle.trustworthiness(X, Y, 15), oracle.trustworthiness(X, Z, 15)
    assert abs(t_many - t_one) < 0.02, (t_many, t_one)


def test_initialize_method_semantics(umap):
    # tests/src/umappp.cpp:209-313
    nn = mock_neighbors(87, 5, seed=87)
    ref = np.zeros((87, 2))
    umap.initialize(csr_tuple(nn), 2, ref)
    assert np.all(ref != 0)
    out = np.zeros((87, 2))
    umap.initialize(csr_tuple(nn), 2, out, umap.Options(initialize_random_on_spectral_fail=False))
    assert np.array_equal(ref, out)
    out = np.zeros((87, 2))
    umap.initialize(csr_tuple(nn), 2, out, umap.Options(initialize_method=umap.InitializeMethod.RANDOM))
    assert np.all(out != 0) and not np.array_equal(ref, out)
    out = np.zeros((87, 2))
    umap.initialize(csr_tuple(nn), 2, out, umap.Options(initialize_method=umap.InitializeMethod.NONE))
    assert np.all(out == 0)

    # spectral failure on two components: random fallback, or untouched without it
    a, b = mock_neighbors(40, 5, seed=40), mock_neighbors(50, 5, seed=50)
    two = oracle.CSR.from_lists(a.to_lists() + [[(j + 40, v) for j, v in r] for r in b.to_lists()])
    ref = np.zeros((90, 2))
    umap.initialize(csr_tuple(two), 2, ref)
    rnd = np.zeros((90, 2))
    umap.initialize(csr_tuple(two), 2, rnd, umap.Options(initialize_method=umap.InitializeMethod.RANDOM))
    assert np.all(ref != 0) and np.array_equal(ref, rnd)
    keep = np.zeros((90, 2))
    umap.initialize(csr_tuple(two), 2, keep, umap.Options(initialize_random_on_spectral_fail=False))
    assert np.all(keep == 0)


def test_float32_path_runs(umap):
    # tests/src/umappp.cpp:150-173
    X = np.random.default_rng(436).normal(size=(87, 7)).astype(np.float32)
    Y = np.zeros((87, 2), np.float32)
    st = umap.initialize_from_data(X, 2, Y, umap.Options(num_neighbors=5))
    st.run(Y)
    assert st.epoch() == 500 and np.all(np.isfinite(Y))


def test_higher_embedding_dimensions(umap):
    X = normal_data(300, 8, seed=3)
    nl = neighbors_of(X, 10)
    for ndim in (1, 3, 5):
        Y = np.zeros((300, ndim))
        st = umap.initialize(csr_tuple(nl), ndim, Y)
        st.run(Y)
        assert np.all(np.isfinite(Y))


def test_invalid_arguments(umap):
    with pytest.raises(umap.UmapbError):
        umap.initialize([[(5, 1.0)], [(0, 1.0)]], 2, np.zeros((2, 2)))   # out-of-range index
    with pytest.raises(umap.UmapbError):
        umap.initialize([[(1, 1.0)], [(0, 1.0)]], 0, np.zeros((2, 0)))  # num_dim 0


def test_cpp_quickstart_runs(umap, tmp_path):
    import subprocess
    from test_capi import _compile_quickstart
    exe = str(tmp_path / "quickstart")
    _compile_quickstart(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "quickstart ok: epochs=500" in r.stdout


def test_knn_matrix_input_matches_neighbor_list(umap):
    """Neighbour matrices with one column per observation (the R harness's
    layout, tests/R/package/src/test.cpp:9-19), 0- or 1-based, host or device,
    give the same state as the same neighbours as a NeighborList."""
    torch = pytest.importorskip("torch")
    X = normal_data(700, 6, seed=31)
    idx, dist = oracle.knn(X, 12)
    ref_Y = np.zeros((700, 2))
    ref = umap.initialize(oracle.CSR.from_dense(idx, dist).to_lists(), 2, ref_Y, umap.Options(num_epochs=30))
    ref_ep = ref.get_epoch_data()
    cases = [(idx, 0), (idx + 1, 1)]
    for ind, base in cases:
        Y = np.zeros((700, 2))
        st = umap.initialize_knn_matrix(ind, dist, 2, Y, umap.Options(num_epochs=30), index_base=base)
        ep = st.get_epoch_data()
        assert np.array_equal(Y, ref_Y)
        assert np.array_equal(ep.edge_targets, ref_ep.edge_targets)
        assert np.array_equal(ep.epochs_per_sample, ref_ep.epochs_per_sample)
    dev = torch.device("cuda", 0)
    d_idx = torch.from_numpy(np.ascontiguousarray(idx, dtype=np.int32)).to(dev)
    d_dist = torch.from_numpy(dist).to(dev)
    Y = np.zeros((700, 2))
    st = umap.initialize_knn_matrix(d_idx, d_dist, 2, Y, umap.Options(num_epochs=30))
    assert np.array_equal(Y, ref_Y) and np.array_equal(st.get_epoch_data().edge_targets, ref_ep.edge_targets)
    st.run(Y)
    assert st.epoch() == 30 and np.all(np.isfinite(Y))


def test_prebuilt_index_matches_data_overload(umap):
    """initialize(const Prebuilt&, ...) (include/umappp/initialize.hpp:138-142):
    a device-resident index searched twice gives the data overload's state."""
    X = normal_data(900, 8, seed=32).astype(np.float32)
    Y_ref = np.zeros((900, 2), np.float32)
    ref = umap.initialize_from_data(X, 2, Y_ref, umap.Options(num_epochs=40))
    pb = umap.Prebuilt(X)
    for _ in range(2):
        Y = np.zeros((900, 2), np.float32)
        st = umap.initialize_prebuilt(pb, 2, Y, umap.Options(num_epochs=40))
        assert np.array_equal(Y, Y_ref)
        assert np.array_equal(st.get_epoch_data().edge_targets, ref.get_epoch_data().edge_targets)
    st.run(Y)
    assert st.epoch() == 40 and np.all(np.isfinite(Y))
