"""The out-of-sample transform on the device (umapb_transform, with its
query-vs-reference search umapb_knn_query) against the oracle's serial
restatement (oracle.transform; the transform has no counterpart in the
reference).

- Search: indices equal to the FP64 brute force except for exchanges of tied
  distances (1e-6 relative); distances the FP64 values rounded to the data's
  type.
- FP64 transform: every row runs the oracle's operations in the same order
  with the same negative-sample stream; the layouts agree to 1e-9 of the
  layout's extent (CUDA's pow and the host's may differ in the last bit).
- FP32 transform: the device uses the hardware power and divide (as the
  layout's epochs do), so positions agree to a looser bound: 99 % of the
  points within 1e-2 of the extent.
- Held-out points of a real layout (an 8-cluster mixture): the reference
  points nearest to a new point in the embedding carry its own cluster's label
  (98 % of the points or more), and the optimisation raises the overlap of its
  15 nearest reference points in the embedding with its 15 nearest in the data
  above that of the similarity-weighted start.
- Repeated calls give identical results; bad arguments are rejected.
"""
import numpy as np
import pytest

import oracle
from helpers import same_neighbors

pytestmark = pytest.mark.gpu


def split(dtype, n=2600, nref=2000, dim=10):
    X = oracle.gaussian_mixture(n, dim, 4, 4.0, seed=11, dtype=dtype)
    return X[:nref], X[nref:]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("k", [5, 15, 40])
def test_knn_query_exact(umap, dtype, k):
    ref, new = split(dtype)
    new = np.vstack([new, ref[:3]])   # queries that coincide with reference points
    idx, dist = umap.knn_query(ref, new, k)
    ridx, rdist = oracle.knn_query(ref, new, k)
    assert same_neighbors(idx, ridx, rdist) == 0
    np.testing.assert_allclose(dist.astype(np.float64), rdist.astype(dtype).astype(np.float64),
                               rtol=1e-6 if dtype == np.float32 else 1e-12, atol=1e-30)
    assert np.all(idx[-3:, 0] == np.arange(3)) and np.all(dist[-3:, 0] == 0)


def reference_layout(dtype, seed=5):
    Y = np.random.default_rng(seed).normal(scale=5.0, size=(2000, 2))
    return Y.astype(dtype)


@pytest.mark.parametrize("dtype,tol,frac", [(np.float64, 1e-9, 1.0), (np.float32, 1e-2, 0.99)])
def test_transform_matches_oracle(umap, dtype, tol, frac):
    ref, new = split(dtype)
    Yref = reference_layout(dtype)
    opt = umap.Options()
    Y = umap.transform(ref, Yref, new, opt, num_epochs=60)
    a, b = oracle.find_ab(1.0, 0.1)
    Yo, init, _, _ = oracle.transform(ref, Yref, new, 15, 60, a, b, seed=opt.optimize_seed)
    extent = float(np.abs(Yref).max())
    err = np.abs(Y.astype(np.float64) - Yo.astype(np.float64)).max(1) / extent
    print(f"{np.dtype(dtype).name}: max error {err.max():.2e} of the extent, median {np.median(err):.2e}, "
          f"moved {np.abs(Yo - init).mean():.3f} on average")
    assert np.mean(err <= tol) >= frac, np.sort(err)[-5:]


def test_transform_repeatable_and_epoch_count(umap):
    ref, new = split(np.float32)
    Yref = reference_layout(np.float32)
    Y1 = umap.transform(ref, Yref, new)
    Y2 = umap.transform(ref, Yref, new)
    assert np.array_equal(Y1, Y2)
    assert umap.transform_epochs(None, 0, len(new)) == 100
    opt = umap.Options(num_epochs=90)
    assert umap.transform_epochs(opt, 0, len(new)) == 30
    assert umap.transform_epochs(opt, 12, len(new)) == 12


def overlap(A, B):
    return np.mean([len(set(a) & set(b)) / len(a) for a, b in zip(A, B)])


def mixture_labels(n, dim, n_clusters, centre_sd, seed):
    """The cluster of every point of oracle.gaussian_mixture(n, dim,
    n_clusters, centre_sd, seed) (equal weights), by the same draws."""
    rng = np.random.default_rng(seed)
    rng.normal(0.0, centre_sd, size=(n_clusters, dim))
    return rng.choice(n_clusters, size=n, p=np.full(n_clusters, 1.0 / n_clusters))


def test_transform_places_held_out_points(umap):
    X = oracle.gaussian_mixture(6000, 20, 8, 4.0, seed=21, dtype=np.float32)
    labels = mixture_labels(6000, 20, 8, 4.0, 21)
    ref, new = X[:5000], X[5000:]
    Yref = np.zeros((5000, 2), np.float32)
    st = umap.initialize_from_data(ref, 2, Yref, umap.Options())
    st.run(Yref)
    Y = umap.transform(ref, Yref, new)
    start = umap.transform(ref, Yref, new, umap.Options(learning_rate=1e-12), num_epochs=1)
    k = 15
    emb_nn, _ = oracle.knn_query(Yref, Y, k)
    votes = labels[:5000][emb_nn]
    placed = np.array([np.bincount(v, minlength=8).argmax() for v in votes])
    accuracy = float(np.mean(placed == labels[5000:]))
    data_nn, _ = oracle.knn_query(ref, new, k)
    start_nn, _ = oracle.knn_query(Yref, start, k)
    final, first = overlap(data_nn, emb_nn), overlap(data_nn, start_nn)
    print(f"cluster placement {accuracy:.4f}; 15-NN overlap with the data: optimised {final:.3f}, start {first:.3f}")
    assert accuracy >= 0.98
    assert final >= first + 0.01


def test_transform_rejects_bad_arguments(umap):
    ref, new = split(np.float32)
    Yref = reference_layout(np.float32)
    with pytest.raises(umap.UmapbError):
        umap.transform(ref[:10], Yref[:10], new, umap.Options(num_neighbors=15))   # k > num_ref
    with pytest.raises(umap.UmapbError):
        umap.transform(ref, Yref, new, umap.Options(learning_rate=0.0))
    assert umap.transform(ref, Yref, new[:0]).shape == (0, 2)
