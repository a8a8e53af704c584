"""Host side of the Python mirror (umappp_b200), without a GPU: the three
neighbour-list forms give the same CSR arrays (the NeighborList of
include/umappp/NeighborList.hpp:24-26 as a list of (index, distance) rows, a
dense (indices, distances) pair as in the R harness, or a CSR triple), and
arguments that cannot be passed to the C ABI are rejected on the host before
any device call: unsupported float types, non-contiguous arrays, foreign
objects, and array shapes that disagree with each other."""
import numpy as np
import pytest

import umappp_b200 as U


def test_neighbor_list_forms_agree():
    rng = np.random.default_rng(4)
    n, k = 7, 3
    idx = np.stack([rng.choice([j for j in range(n) if j != i], size=k, replace=False) for i in range(n)])
    dist = np.sort(rng.random((n, k)), axis=1)
    rows = [[(int(idx[i, c]), float(dist[i, c])) for c in range(k)] for i in range(n)]
    a = U.to_csr(rows)
    b = U.to_csr((idx, dist))
    c = U.to_csr((np.arange(n + 1) * k, idx.reshape(-1), dist.reshape(-1)))
    for x, y in ((a, b), (a, c)):
        assert x[0].dtype == np.int64 and x[1].dtype == np.int32
        for u, v in zip(x, y):
            assert np.array_equal(u, v)
    # ragged rows, an empty row, and the value type on request
    p, i, v = U.to_csr([[(1, 0.5), (2, 1.0)], [], [(0, 0.25)]], dtype=np.float32)
    assert p.tolist() == [0, 2, 2, 3] and i.tolist() == [1, 2, 0] and v.dtype == np.float32


def test_unsupported_types_are_rejected():
    for dt in (np.float16, np.int32, np.complex64):
        with pytest.raises(TypeError):
            U._dtype_code(dt)
    with pytest.raises(ValueError):
        U._ptr(np.zeros((4, 4), np.float32)[:, ::2])
    with pytest.raises(TypeError):
        U._ptr([1.0, 2.0])
    with pytest.raises(TypeError):
        U._float_dtype(12345)
    assert U._ptr(None) is None and U._ptr(4096) == 4096


def test_disagreeing_shapes_are_rejected_on_the_host():
    x = np.zeros((10, 3), np.float32)
    with pytest.raises(ValueError, match="sum"):
        U.batch_run(x, [4, 5], 2, np.zeros((10, 2), np.float32))
    with pytest.raises(ValueError, match="columns"):
        U.knn_query(x, np.zeros((4, 2), np.float32), 3)
    with pytest.raises(ValueError, match="one row per reference"):
        U.transform(x, np.zeros((9, 2), np.float32), np.zeros((2, 3), np.float32))
    with pytest.raises(ValueError, match="columns"):
        U.transform(x, np.zeros((10, 2), np.float32), np.zeros((2, 4), np.float32))


def test_options_reach_the_c_struct():
    o = U.Options(num_neighbors=30, num_epochs=77, learning_rate=0.5, negative_sample_rate=7,
                  mix_ratio=0.25, local_connectivity=2.0, optimize_seed=42)
    c = o.to_c()
    assert c.num_neighbors == 30 and c.num_epochs == 77
    assert c.learning_rate == 0.5 and c.negative_sample_rate == 7
    assert c.mix_ratio == 0.25 and c.local_connectivity == 2.0 and c.optimize_seed == 42


def test_transform_epoch_rule_without_a_device():
    # 100 epochs up to 10,000 new points, 30 above, unless a count is given
    assert U.transform_epochs(None, 0, 1) == 100
    assert U.transform_epochs(None, 0, 10_000) == 100
    assert U.transform_epochs(None, 0, 10_001) == 30
    assert U.transform_epochs(None, 57, 20_000) == 57
