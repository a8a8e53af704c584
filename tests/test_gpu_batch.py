"""Batched runs (umapb_batch_run): many independent UMAP instances in one pass.

Each instance must get what initialize_from_data + run give it alone: the
same neighbours, weights, union, initial layout (exactly, up to rounding of
the spectral solver) and a layout of the same quality.  Negative samples stay
inside their instance, so instances do not push each other around.
"""
import numpy as np
import pytest

import oracle
from helpers import normal_data, two_populations

pytestmark = pytest.mark.gpu


def _split(Y, sizes):
    return np.split(Y, np.cumsum(sizes)[:-1])


def _instances(sizes, dim, dtype, seed):
    parts = []
    for i, m in enumerate(sizes):
        if i % 3 == 2:
            parts.append(two_populations(m, dim, seed=seed + i, dtype=dtype))   # two components: spectral fails
        else:
            parts.append(oracle.gaussian_mixture(m, dim, 4, 4.0, seed=seed + i, dtype=dtype))
    return parts


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("method", ["spectral", "random"])
def test_initial_layouts_match_single_runs(umap, dtype, method):
    # learning rate 0: the epochs run (graph capture, tuned launch shape) but move nothing
    sizes = [11, 127, 128, 129, 400, 1000, 260]
    dim = 10
    parts = _instances(sizes, dim, dtype, seed=70)
    X = np.ascontiguousarray(np.concatenate(parts))
    m = umap.InitializeMethod.SPECTRAL if method == "spectral" else umap.InitializeMethod.RANDOM
    opt = umap.Options(num_neighbors=10, num_epochs=20, learning_rate=0.0, initialize_method=m)
    Y = np.zeros((len(X), 2), dtype=dtype)
    ms = umap.batch_run(X, sizes, 2, Y, opt)
    assert set(ms) == {"knn", "similarities", "union", "init", "epochs", "schedule", "sgd"}
    rtol = 1e-9 if dtype == np.float64 else 1e-4
    for Xi, Yb in zip(parts, _split(Y, sizes)):
        Ys = np.zeros((len(Xi), 2), dtype=dtype)
        st = umap.initialize_from_data(Xi, 2, Ys, opt)
        st.run(Ys)
        assert np.all(Ys != 0)
        scale = np.max(np.abs(Ys))
        assert np.max(np.abs(Yb - Ys)) <= rtol * scale, (len(Xi), np.max(np.abs(Yb - Ys)), scale)


def test_initialize_none_keeps_the_given_layouts(umap):
    sizes = [50, 70]
    X = normal_data(120, 5, seed=4)
    Y0 = np.random.default_rng(5).normal(size=(120, 2))
    Y = Y0.copy()
    umap.batch_run(X, sizes, 2, Y, umap.Options(initialize_method=umap.InitializeMethod.NONE,
                                                num_epochs=10, learning_rate=0.0))
    assert np.array_equal(Y, Y0)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_layout_quality_matches_single_runs(umap, dtype):
    sizes = [600, 1500, 2500]
    dim = 20
    parts = [oracle.gaussian_mixture(m, dim, 5, 5.0, seed=300 + i, dtype=dtype) for i, m in enumerate(sizes)]
    X = np.ascontiguousarray(np.concatenate(parts))
    Y = np.zeros((len(X), 2), dtype=dtype)
    umap.batch_run(X, sizes, 2, Y, umap.Options())
    assert np.all(np.isfinite(Y))
    for Xi, Yb in zip(parts, _split(Y, sizes)):
        Ys = np.zeros((len(Xi), 2), dtype=dtype)
        st = umap.initialize_from_data(Xi, 2, Ys, umap.Options())
        st.run(Ys)
        tb, ts = oracle.trustworthiness(Xi, Yb, 15), oracle.trustworthiness(Xi, Ys, 15)
        # a single run's trustworthiness varies by ~0.007 from seed to seed at these sizes
        assert abs(tb - ts) <= 0.02, (len(Xi), tb, ts)


def test_instances_do_not_interact(umap):
    # two copies of one instance, the second moved far away in data space:
    # both layouts must be as good as a single run's (cross-instance
    # neighbours or negatives would tie the copies together)
    A = two_populations(400, 5, seed=12)
    X = np.concatenate([A, A + 1000.0])
    Y = np.zeros((800, 2))
    umap.batch_run(X, [400, 400], 2, Y, umap.Options())
    for Yb in _split(Y, [400, 400]):
        even, odd = Yb[0::2], Yb[1::2]
        assert any(even[:, d].max() < odd[:, d].min() or odd[:, d].max() < even[:, d].min() for d in range(2))
        assert oracle.trustworthiness(A, Yb, 15) > 0.9


def test_many_instances(umap):
    # log-uniform sizes, 30 dimensions, float32: the batched workload's shape at 1/8 scale
    rng = np.random.default_rng(64)
    sizes = np.exp(rng.uniform(np.log(100), np.log(3000), size=64)).astype(np.int32)
    parts = [oracle.gaussian_mixture(int(m), 30, 5, 5.0, seed=500 + i) for i, m in enumerate(sizes)]
    X = np.ascontiguousarray(np.concatenate(parts))
    Y = np.zeros((len(X), 2), dtype=np.float32)
    opt = umap.Options(num_epochs=200)
    umap.batch_run(X, sizes, 2, Y, opt)
    assert np.all(np.isfinite(Y))
    blocks = _split(Y, sizes)
    for i in (0, 17, int(np.argmax(sizes)), int(np.argmin(sizes))):
        Ys = np.zeros((sizes[i], 2), dtype=np.float32)
        st = umap.initialize_from_data(parts[i], 2, Ys, opt)
        st.run(Ys)
        tb, ts = oracle.trustworthiness(parts[i], blocks[i], 15), oracle.trustworthiness(parts[i], Ys, 15)
        assert abs(tb - ts) <= 0.03, (int(sizes[i]), tb, ts)


def test_invalid_batches(umap):
    X = normal_data(20100, 3, seed=1)
    Y = np.zeros((20100, 2))
    with pytest.raises(umap.UmapbError, match="epoch"):
        umap.batch_run(X, [100, 20000], 2, Y)                     # 500 vs 215 epochs
    with pytest.raises(umap.UmapbError):
        umap.batch_run(X[:110], [10, 100], 2, Y[:110])            # 10 <= num_neighbors
    with pytest.raises(ValueError):
        umap.batch_run(X[:110], [50, 50], 2, Y[:110])             # rows != sum(sizes)
