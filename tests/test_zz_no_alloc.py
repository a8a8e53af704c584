"""The allocation-free adjoint entry point, umapb_loss_grad_noalloc.

It is for callers that cannot call cudaMalloc (a framework that owns all device
memory through its own pool, or a serving loop whose request path must not
block on the allocator): it keeps its scratch in a fixed array of the
library's device memory instead of allocating.  This test calls it through the
C ABI with device buffers, twice in a row (the second call reuses the scratch
the first one left behind), and checks each result against the regular entry
point umapb_loss_grad within the tolerances of the other adjoint tests
(1e-10 relative for FP64, 1e-6 for FP32).  It runs last in the suite (file
name) and also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import oracle
from helpers import csr_tuple, neighbors_of, normal_data

pytestmark = pytest.mark.gpu


def _noalloc_fn(umap):
    L = umap._lib.lib()
    fn = L.umapb_loss_grad_noalloc
    v = ctypes.c_void_p
    fn.argtypes = [ctypes.c_int, ctypes.c_size_t, v, ctypes.c_int32, v, v, v, ctypes.c_double, ctypes.c_double,
                   ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double), v, v]
    fn.restype = ctypes.c_int
    return fn


def _problem(dtype):
    nl = neighbors_of(normal_data(400, 6, seed=21), 10)
    w, _, _ = oracle.neighbor_similarities(nl)
    g = oracle.combine_neighbor_sets(w, 1.0).astype(dtype)
    Y = (np.random.default_rng(3).normal(size=(400, 2)) * 3).astype(dtype)
    return g, Y


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_noalloc_matches_regular_entry_point(umap, dtype):
    torch = pytest.importorskip("torch")
    fn = _noalloc_fn(umap)
    g, Y = _problem(dtype)
    a, b = oracle.find_ab(1.0, 0.1)
    code = 1 if dtype == np.float64 else 0
    tol = 1e-10 if dtype == np.float64 else 1e-6
    ref_loss, ref_grad, ref_ab = umap.loss_grad(csr_tuple(g), Y, a, b, eps_rep=0.001, with_constant=True)

    dev = torch.device("cuda", 0)
    d_Y = torch.from_numpy(Y).to(dev)
    d_ptr = torch.from_numpy(g.ptr).to(dev)
    d_idx = torch.from_numpy(g.idx).to(dev)
    d_w = torch.from_numpy(g.val).to(dev)
    torch.cuda.synchronize()
    for call in range(2):
        d_grad = torch.full(Y.shape, float("nan"), dtype=d_Y.dtype, device=dev)   # must be fully overwritten
        torch.cuda.synchronize()
        loss = ctypes.c_double()
        gab = np.zeros(2, dtype=np.float64)
        rc = fn(code, 2, d_Y.data_ptr(), g.n, d_ptr.data_ptr(), d_idx.data_ptr(), d_w.data_ptr(), a, b, 0.001, 1,
                ctypes.byref(loss), d_grad.data_ptr(), gab.ctypes.data)
        assert rc == 0, umap._lib.lib().umapb_last_error().decode()
        grad = d_grad.cpu().numpy()
        assert abs(loss.value - ref_loss) <= tol * abs(ref_loss), (call, loss.value, ref_loss)
        assert np.max(np.abs(grad - ref_grad)) <= tol * np.max(np.abs(ref_grad)), call
        assert np.max(np.abs(gab - np.array(ref_ab))) <= tol * np.max(np.abs(ref_ab)), call


def test_noalloc_rejects_host_pointers_and_oversize(umap):
    torch = pytest.importorskip("torch")
    fn = _noalloc_fn(umap)
    g, Y = _problem(np.float32)
    loss = ctypes.c_double()
    # host arrays are refused (the entry point cannot stage them without allocating)
    rc = fn(0, 2, Y.ctypes.data, g.n, g.ptr.ctypes.data, g.idx.ctypes.data, g.val.ctypes.data, 1.5, 0.9, 0.0, 0,
            ctypes.byref(loss), None, None)
    assert rc == 1 and "device pointers" in umap._lib.lib().umapb_last_error().decode()
    # a float gradient above the scratch's 4194304 elements is refused before any device work
    dev = torch.device("cuda", 0)
    d_Y = torch.zeros((8, 2), dtype=torch.float32, device=dev)
    d_ptr = torch.zeros(9, dtype=torch.int64, device=dev)
    d_idx = torch.zeros(1, dtype=torch.int32, device=dev)
    d_w = torch.zeros(1, dtype=torch.float32, device=dev)
    d_g = torch.zeros((8, 2), dtype=torch.float32, device=dev)
    rc = fn(0, 2, d_Y.data_ptr(), 3_000_000, d_ptr.data_ptr(), d_idx.data_ptr(), d_w.data_ptr(), 1.5, 0.9, 0.0, 0,
            ctypes.byref(loss), d_g.data_ptr(), None)
    assert rc == 1 and "scratch" in umap._lib.lib().umapb_last_error().decode()


def test_noalloc_rejects_bad_indices_and_accepts_empty(umap):
    """An index outside [0, num_obs) or a row_ptr running backwards is found on
    the device (the bad edges are skipped, never read) and reported as
    UMAPB_ERR_INVALID; a following valid call succeeds.  num_obs == 0 reads
    no pointer at all."""
    torch = pytest.importorskip("torch")
    fn = _noalloc_fn(umap)
    g, Y = _problem(np.float64)
    a, b = oracle.find_ab(1.0, 0.1)
    dev = torch.device("cuda", 0)
    d_Y = torch.from_numpy(Y).to(dev)
    d_w = torch.from_numpy(g.val).to(dev)
    loss = ctypes.c_double()
    bad_idx = g.idx.copy()
    bad_idx[len(bad_idx) // 2] = g.n          # one neighbour out of range
    bad_ptr = g.ptr.copy()
    bad_ptr[5] = bad_ptr[7]                   # row 5 runs backwards
    for ptr, idx in ((g.ptr, bad_idx), (bad_ptr, g.idx)):
        d_ptr = torch.from_numpy(ptr).to(dev)
        d_idx = torch.from_numpy(idx).to(dev)
        rc = fn(1, 2, d_Y.data_ptr(), g.n, d_ptr.data_ptr(), d_idx.data_ptr(), d_w.data_ptr(), a, b, 0.001, 0,
                ctypes.byref(loss), None, None)
        assert rc == 1 and "out of range" in umap._lib.lib().umapb_last_error().decode()
    d_ptr = torch.from_numpy(g.ptr).to(dev)
    d_idx = torch.from_numpy(g.idx).to(dev)
    rc = fn(1, 2, d_Y.data_ptr(), g.n, d_ptr.data_ptr(), d_idx.data_ptr(), d_w.data_ptr(), a, b, 0.001, 0,
            ctypes.byref(loss), None, None)
    assert rc == 0
    ref_loss, _, _ = umap.loss_grad(csr_tuple(g), Y, a, b, eps_rep=0.001)
    assert abs(loss.value - ref_loss) <= 1e-10 * abs(ref_loss)
    gab = np.full(2, np.nan)
    rc = fn(1, 2, None, 0, None, None, None, a, b, 0.001, 0, ctypes.byref(loss), None, gab.ctypes.data)
    assert rc == 0 and loss.value == 0 and np.all(gab == 0)
