"""Failure paths, made to happen without faulting the GPU.

- A bounded device wait that runs out: the tensor-core kNN's mbarrier waits
  take their poll limit from umapb_set_device_wait_limit; with a limit of one
  poll the first wait for a TMA copy gives up, the kernel stops every role,
  waits for its copies and MMAs in flight, frees its tensor memory and the call
  returns UMAPB_ERR_DEVICE_TIMEOUT.  The next call, with the default limit,
  must succeed and be exact.
- Out of device memory: umapb_set_workspace_limit caps what the library may
  hold; a pipeline run beyond the cap fails with UMAPB_ERR_OOM, and the same
  run succeeds once the cap is lifted.
- The spectral eigensolver not converging (irlba's max_iterations = 1 on a
  connected graph): initialize() falls back to the random layout, or leaves
  the embedding untouched when initialize_random_on_spectral_fail is false
  (include/umappp/initialize.hpp:79-103; spectral_init.hpp:122-125).
"""
import numpy as np
import pytest

import oracle
from helpers import csr_tuple, mock_neighbors, same_neighbors

pytestmark = pytest.mark.gpu

ERR_OOM, ERR_DEVICE_TIMEOUT = 2, 4


def test_device_wait_timeout_then_recovery(umap):
    L = umap.lib()
    X = oracle.gaussian_mixture(3000, 20, 4, 3.0, seed=9, dtype=np.float32)
    prev = L.umapb_set_device_wait_limit(1)
    try:
        with pytest.raises(umap.UmapbError) as ei:
            umap.knn(X, 15)
        assert ei.value.code == ERR_DEVICE_TIMEOUT
    finally:
        L.umapb_set_device_wait_limit(prev)
    idx, dist = umap.knn(X, 15)
    ridx, rdist = oracle.knn(X, 15)
    assert same_neighbors(idx, ridx, rdist) == 0


def test_workspace_limit_gives_oom_then_recovery(umap):
    L = umap.lib()
    X = oracle.gaussian_mixture(5000, 16, 4, 3.0, seed=10, dtype=np.float32)
    opt = umap.Options(num_epochs=20)
    prev = L.umapb_set_workspace_limit(1 << 20)
    try:
        with pytest.raises(umap.UmapbError) as ei:
            Y = np.zeros((5000, 2), np.float32)
            umap.initialize_from_data(X, 2, Y, opt).run(Y)
        assert ei.value.code == ERR_OOM and "workspace limit" in str(ei.value)
    finally:
        L.umapb_set_workspace_limit(prev)
    Y = np.zeros((5000, 2), np.float32)
    st = umap.initialize_from_data(X, 2, Y, opt)
    st.run(Y)
    assert st.epoch() == 20 and np.all(np.isfinite(Y))


def test_spectral_nonconvergence_falls_back(umap):
    nn = mock_neighbors(500, 10, seed=77)   # connected (forced chain)
    assert not oracle.has_multiple_components(oracle.combine_neighbor_sets(oracle.neighbor_similarities(nn)[0]))
    stuck = umap.IrlbaOptions(max_iterations=1, convergence_tolerance=1e-14)
    spectral = np.zeros((500, 2))
    umap.initialize(csr_tuple(nn), 2, spectral)
    rnd = np.zeros((500, 2))
    umap.initialize(csr_tuple(nn), 2, rnd, umap.Options(initialize_method=umap.InitializeMethod.RANDOM))
    out = np.zeros((500, 2))
    umap.initialize(csr_tuple(nn), 2, out, umap.Options(initialize_spectral_irlba_options=stuck))
    assert np.array_equal(out, rnd) and not np.array_equal(spectral, rnd)
    keep = np.zeros((500, 2))
    umap.initialize(csr_tuple(nn), 2, keep, umap.Options(initialize_spectral_irlba_options=stuck,
                                                          initialize_random_on_spectral_fail=False))
    assert np.all(keep == 0)
