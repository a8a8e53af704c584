"""The transform oracle (oracle.transform, no counterpart in the reference:
it restates the device's umapb_transform), checked on the CPU:

- the negative-sample stream (Philox4x32-7 with Lemire's bounded integers,
  restated in oracle.c) against an independent pure-Python restatement of the
  same published algorithms;
- the query-vs-reference FP64 search against a numpy brute force;
- the starting positions against a vectorised weighted mean;
- the epoch-count rule, and that zero-weight-free rows keep their k edges.
"""
import numpy as np
import pytest

import oracle

M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32_7(c, k0, k1):
    c0, c1, c2, c3 = c
    for _ in range(7):
        p0, p1 = M0 * c0, M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & MASK, p1 & MASK, ((p0 >> 32) ^ c3 ^ k1) & MASK, p0 & MASK
        k0, k1 = (k0 + W0) & MASK, (k1 + W1) & MASK
    return [c0, c1, c2, c3]


def py_draws(head, tail, epoch, seed, n, count):
    k0 = (seed & MASK) ^ 0x4E454731
    k1 = (seed >> 32) & MASK
    block, buf, out = 0, [], []

    def nxt():
        nonlocal block, buf
        if not buf:
            buf = philox4x32_7([head, tail, epoch, block], k0, k1)
            block += 1
        return buf.pop(0)

    for _ in range(count):
        m = nxt() * n
        if (m & MASK) < n:
            thr = ((1 << 32) - n) % n
            while (m & MASK) < thr:
                m = nxt() * n
        out.append(m >> 32)
    return out


@pytest.mark.parametrize("head,tail,epoch,seed,n", [(0, 0, 0, 1234567890, 1000), (12345, 678, 99, 2**40 + 17, 7),
                                                    (2**31 - 1, 5, 1, 0, 3_000_000), (3, 4, 5, 99, 1)])
def test_negative_stream_matches_independent_restatement(oracle_mod, head, tail, epoch, seed, n):
    got = oracle.negstream_draws(head, tail, epoch, seed, n, 41)
    assert got.tolist() == py_draws(head, tail, epoch, seed, n, 41)
    assert np.all((got >= 0) & (got < n))


def test_query_knn_matches_brute_force(oracle_mod):
    rng = np.random.default_rng(1)
    ref = rng.normal(size=(400, 6))
    ref[10] = ref[11]          # an exact duplicate: ties go to the smaller index
    q = np.vstack([rng.normal(size=(50, 6)), ref[10:11]])
    idx, dist = oracle.knn_query(ref, q, 9)
    d2 = ((q[:, None, :] - ref[None, :, :]) ** 2).sum(-1)
    order = np.lexsort((np.broadcast_to(np.arange(400), d2.shape), d2), axis=-1)[:, :9]
    assert np.array_equal(idx, order)
    np.testing.assert_allclose(dist, np.sqrt(np.take_along_axis(d2, order, 1)), rtol=1e-12)
    assert idx[-1, 0] == 10 and idx[-1, 1] == 11 and dist[-1, 0] == 0.0


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_transform_start_and_schedule(oracle_mod, dtype):
    X = oracle.gaussian_mixture(700, 8, 3, 4.0, seed=3, dtype=dtype)
    Yref = np.random.default_rng(2).normal(size=(600, 2)).astype(dtype)
    a, b = oracle.find_ab(1.0, 0.1)
    Y, init, idx, w = oracle.transform(X[:600], Yref, X[600:], 15, 30, a, b)
    wv = w.val.astype(np.float64).reshape(100, 15)
    want = (wv[:, :, None] * Yref[idx].astype(np.float64)).sum(1) / wv.sum(1)[:, None]
    np.testing.assert_allclose(init.astype(np.float64), want, rtol=1e-5 if dtype == np.float32 else 1e-12)
    assert np.all(np.isfinite(Y)) and Y.dtype == dtype
    assert np.all(np.diff(w.ptr) == 15)
    # the new points move, and stay near the reference layout's range
    assert np.abs(Y - init).max() > 0
    assert np.abs(Y).max() < 10 * np.abs(Yref).max()


def test_transform_epoch_rule(oracle_mod):
    assert oracle.transform_epochs(7, True, 500, 50) == 7
    assert oracle.transform_epochs(0, True, 500, 50) == 166
    assert oracle.transform_epochs(0, False, 0, 10000) == 100
    assert oracle.transform_epochs(0, False, 0, 10001) == 30
