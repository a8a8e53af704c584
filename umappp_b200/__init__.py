"""umappp_b200 -- UMAP on B200 GPUs behind the umappp interface.

Python mirror of the reference's API (libscran/umappp v3.3.2,
include/umappp/*.hpp), calling the CUDA library libumappp_b200.so through its
C ABI (include/umapb.h):

    opt = Options(num_epochs=200)
    status = initialize(neighbors, 2, embedding, opt)   # initialize.hpp:69-119
    status.run(embedding)                               # Status.hpp:101-140

    status = initialize_from_data(data, 2, embedding, opt)   # initialize.hpp:165-177, exact device kNN

Arrays are NumPy (host) arrays, or any object exposing
``__cuda_array_interface__`` (device memory; used in place), or raw device
pointers given as ints.  Layouts are the reference's: observation i of a data
or embedding matrix occupies row i of an (n, dim) C-ordered array
(column-major with observations as columns in the reference's terms).
Neighbour lists are a list of lists of (index, distance) pairs (the
reference's NeighborList), a dense (indices, distances) pair of (n, k)
arrays, or a CSR triple (row_ptr, indices, values).  The stage functions of
the reference are exposed with the same names.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib
from ._lib import F32, F64, UmapbError, check, lib

__all__ = [
    "InitializeMethod", "Options", "Status", "EpochData", "initialize", "initialize_from_data", "knn",
    "neighbor_similarities", "combine_neighbor_sets", "similarities_to_epochs", "has_multiple_components",
    "spectral_init", "random_init", "find_ab", "choose_num_epochs", "optimize_layout", "loss_grad", "UmapbError",
    "to_csr", "batch_run", "initialize_knn_matrix", "Prebuilt", "initialize_prebuilt", "knn_shard",
    "knn_query", "transform", "transform_epochs",
]


class InitializeMethod(enum.IntEnum):
    """include/umappp/Options.hpp:27."""

    SPECTRAL = 0
    RANDOM = 1
    NONE = 2


@dataclass
class IrlbaOptions:
    """Stands in for irlba::Options (Options.hpp:110): the spectral eigensolver's knobs."""

    extra_work: int = 7
    max_iterations: int = 1000
    convergence_tolerance: float = 1e-6


@dataclass
class Options:
    """include/umappp/Options.hpp:37-218, field for field (num_threads* are accepted and ignored)."""

    local_connectivity: float = 1.0
    bandwidth: float = 1.0
    mix_ratio: float = 1.0
    spread: float = 1.0
    min_dist: float = 0.1
    a: Optional[float] = None
    b: Optional[float] = None
    repulsion_strength: float = 1.0
    initialize_method: InitializeMethod = InitializeMethod.SPECTRAL
    initialize_random_on_spectral_fail: bool = True
    initialize_spectral_irlba_options: IrlbaOptions = field(default_factory=IrlbaOptions)
    initialize_spectral_scale: float = 10.0
    initialize_spectral_jitter: bool = False
    initialize_spectral_jitter_sd: float = 1e-4
    initialize_random_scale: float = 10.0
    initialize_seed: int = 9876543210
    num_epochs: Optional[int] = None
    learning_rate: float = 1.0
    negative_sample_rate: float = 5.0
    num_neighbors: int = 15
    optimize_seed: int = 1234567890
    num_threads: int = 1
    num_threads_spectral: int = 1
    num_threads_optimize: int = 1

    def to_c(self) -> _lib.UmapbOptions:
        o = _lib.UmapbOptions()
        lib().umapb_options_init(ctypes.byref(o))
        for name in ("local_connectivity", "bandwidth", "mix_ratio", "spread", "min_dist", "repulsion_strength",
                     "initialize_spectral_scale", "initialize_spectral_jitter_sd", "initialize_random_scale",
                     "learning_rate", "negative_sample_rate"):
            setattr(o, name, float(getattr(self, name)))
        o.has_a, o.a = (0, 0.0) if self.a is None else (1, float(self.a))
        o.has_b, o.b = (0, 0.0) if self.b is None else (1, float(self.b))
        o.initialize_method = int(self.initialize_method)
        o.initialize_random_on_spectral_fail = int(bool(self.initialize_random_on_spectral_fail))
        o.irlba_extra_work = int(self.initialize_spectral_irlba_options.extra_work)
        o.irlba_max_iterations = int(self.initialize_spectral_irlba_options.max_iterations)
        o.irlba_convergence_tolerance = float(self.initialize_spectral_irlba_options.convergence_tolerance)
        o.initialize_spectral_jitter = int(bool(self.initialize_spectral_jitter))
        o.initialize_seed = int(self.initialize_seed)
        o.has_num_epochs, o.num_epochs = (0, 0) if self.num_epochs is None else (1, int(self.num_epochs))
        o.num_neighbors = int(self.num_neighbors)
        o.optimize_seed = int(self.optimize_seed)
        o.num_threads, o.num_threads_spectral, o.num_threads_optimize = (
            int(self.num_threads), int(self.num_threads_spectral), int(self.num_threads_optimize))
        return o


# ----------------------------------------------------------------- arrays --

def _dtype_code(dtype) -> int:
    dt = np.dtype(dtype)
    if dt == np.float32:
        return F32
    if dt == np.float64:
        return F64
    raise TypeError(f"unsupported float type {dt}; use float32 or float64")


def _ptr(x):
    """Address of a host NumPy array, a __cuda_array_interface__ object or an int device pointer."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        if not x.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return x.ctypes.data
    cai = getattr(x, "__cuda_array_interface__", None)
    if cai is not None:
        return int(cai["data"][0])
    raise TypeError(f"cannot pass {type(x)} to the device library")


def _float_dtype(x) -> np.dtype:
    if isinstance(x, np.ndarray):
        return x.dtype
    cai = getattr(x, "__cuda_array_interface__", None)
    if cai is not None:
        return np.dtype(cai["typestr"])
    raise TypeError("cannot infer the float type of a raw pointer")


def to_csr(neighbors, dtype=None):
    """NeighborList (list of lists of pairs), dense (indices, distances) or CSR triple -> host CSR arrays."""
    if isinstance(neighbors, tuple) and len(neighbors) == 3:
        ptr, idx, val = neighbors
        return (np.ascontiguousarray(ptr, dtype=np.int64), np.ascontiguousarray(idx, dtype=np.int32),
                np.ascontiguousarray(val, dtype=dtype or np.asarray(val).dtype))
    if isinstance(neighbors, tuple) and len(neighbors) == 2:
        idx, dist = (np.asarray(a) for a in neighbors)
        n, k = idx.shape
        return (np.arange(n + 1, dtype=np.int64) * k, np.ascontiguousarray(idx.reshape(-1), dtype=np.int32),
                np.ascontiguousarray(dist.reshape(-1), dtype=dtype or dist.dtype))
    rows = list(neighbors)
    ptr = np.zeros(len(rows) + 1, dtype=np.int64)
    for i, r in enumerate(rows):
        ptr[i + 1] = ptr[i] + len(r)
    idx = np.fromiter((j for r in rows for j, _ in r), dtype=np.int32, count=int(ptr[-1]))
    val = np.fromiter((v for r in rows for _, v in r), dtype=dtype or np.float64, count=int(ptr[-1]))
    return ptr, idx, val


# ----------------------------------------------------------------- status --

@dataclass
class EpochData:
    """include/umappp/optimize_layout.hpp:27-45 as arrays (at the status' current epoch)."""

    cumulative_num_edges: np.ndarray
    edge_targets: np.ndarray
    epochs_per_sample: np.ndarray
    epoch_of_next_sample: np.ndarray
    epoch_of_next_negative_sample: np.ndarray
    total_epochs: int
    current_epoch: int


STAGES = ("knn", "similarities", "union", "init", "epochs", "schedule", "sgd")


class Status:
    """include/umappp/Status.hpp:25-141 over a device-resident state."""

    def __init__(self, handle: int, dtype):
        self._h = ctypes.c_void_p(handle)
        self.dtype = np.dtype(dtype)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().umapb_status_free(h)
            except Exception:   # interpreter shutdown: module globals already gone
                pass
            self._h = None

    def run(self, embedding, epoch_limit: Optional[int] = None) -> None:
        """Status::run(embedding, epoch_limit) / Status::run(embedding)."""
        check(lib().umapb_status_run(self._h, _ptr(embedding), -1 if epoch_limit is None else int(epoch_limit)))

    def epoch(self) -> int:
        return lib().umapb_status_epoch(self._h)

    def num_epochs(self) -> int:
        return lib().umapb_status_num_epochs(self._h)

    def num_observations(self) -> int:
        return lib().umapb_status_num_observations(self._h)

    def num_dimensions(self) -> int:
        return lib().umapb_status_num_dimensions(self._h)

    @property
    def a(self) -> float:
        return lib().umapb_status_a(self._h)

    @property
    def b(self) -> float:
        return lib().umapb_status_b(self._h)

    def num_edges(self) -> int:
        return lib().umapb_status_num_edges(self._h)

    def get_epoch_data(self) -> EpochData:
        n = self.num_observations()
        nnz = self.num_edges()
        ptr = np.zeros(n + 1, dtype=np.int64)
        tg = np.zeros(max(nnz, 1), dtype=np.int32)
        arrs = [np.zeros(max(nnz, 1), dtype=self.dtype) for _ in range(3)]
        check(lib().umapb_status_get_epoch_data(self._h, _ptr(ptr), _ptr(tg), *(_ptr(a) for a in arrs)))
        return EpochData(ptr, tg[:nnz], *(a[:nnz] for a in arrs), total_epochs=self.num_epochs(),
                         current_epoch=self.epoch())

    def schedule_counts(self, first: int = 0, last: Optional[int] = None) -> np.ndarray:
        """(epochs, 2) array of [firing edges, negative samples drawn] per epoch."""
        last = self.num_epochs() if last is None else last
        out = np.zeros((max(last - first, 0), 2), dtype=np.int64)
        if last > first:
            check(lib().umapb_status_schedule_counts(self._h, first, last, _ptr(out)))
        return out

    def stage_ms(self) -> dict:
        ms = np.zeros(len(STAGES), dtype=np.float64)
        check(lib().umapb_status_stage_ms(self._h, _ptr(ms), len(STAGES)))
        return dict(zip(STAGES, ms.tolist()))


def initialize(neighbors, num_dim: int, embedding, options: Optional[Options] = None, dtype=None) -> Status:
    """initialize(NeighborList x, num_dim, embedding, Options) (include/umappp/initialize.hpp:69-119).
    A dense (indices, distances) pair of (n, k) arrays -- the k x n
    column-per-observation matrices of the reference's R harness, in memory --
    goes to the device as it is (initialize_knn_matrix)."""
    options = options or Options()
    dt = np.dtype(dtype) if dtype is not None else _float_dtype(embedding)
    if isinstance(neighbors, tuple) and len(neighbors) == 2:
        idx, dist = neighbors
        return initialize_knn_matrix(idx, np.asarray(dist, dtype=dt), num_dim, embedding, options)
    ptr, idx, val = to_csr(neighbors, dt)
    n = len(ptr) - 1
    out = ctypes.c_void_p()
    copt = options.to_c()
    check(lib().umapb_initialize_neighbors(_dtype_code(dt), n, _ptr(ptr), _ptr(idx), _ptr(val), num_dim,
                                           _ptr(embedding), ctypes.byref(copt), ctypes.byref(out)))
    return Status(out.value, dt)


def initialize_knn_matrix(indices, distances, num_dim: int, embedding, options: Optional[Options] = None,
                          index_base: int = 0, num_obs: Optional[int] = None, k: Optional[int] = None) -> Status:
    """initialize(NeighborList, ...) from neighbour matrices with one column per
    observation (k x n column-major = (n, k) C-ordered: row i holds observation
    i's neighbours by increasing distance), the R harness's layout
    (tests/R/package/src/test.cpp:9-19); index_base=1 for R's 1-based indices.
    Arrays may be host or device memory; for device pointers give num_obs and k."""
    options = options or Options()
    dt = _float_dtype(distances) if not isinstance(distances, int) else _float_dtype(embedding)
    if isinstance(indices, np.ndarray):
        indices = np.ascontiguousarray(indices, dtype=np.int32)
    if isinstance(distances, np.ndarray):
        distances = np.ascontiguousarray(distances)
    if num_obs is None or k is None:
        shape = indices.shape if isinstance(indices, np.ndarray) else tuple(indices.__cuda_array_interface__["shape"])
        num_obs, k = int(shape[0]), int(shape[1])
    out = ctypes.c_void_p()
    copt = options.to_c()
    check(lib().umapb_initialize_knn_matrix(_dtype_code(dt), num_obs, k, _ptr(indices), _ptr(distances),
                                            int(index_base), num_dim, _ptr(embedding), ctypes.byref(copt),
                                            ctypes.byref(out)))
    return Status(out.value, dt)


class Prebuilt:
    """A neighbour-search index resident on the device (knncolle::Prebuilt's
    role, include/umappp/initialize.hpp:138-142): the data copied to the
    current device once, searched by every initialize_prebuilt."""

    def __init__(self, data, num_obs: Optional[int] = None, data_dim: Optional[int] = None):
        self.dtype = _float_dtype(data)
        if num_obs is None or data_dim is None:
            shape = data.shape if isinstance(data, np.ndarray) else tuple(data.__cuda_array_interface__["shape"])
            num_obs, data_dim = int(shape[0]), int(shape[1])
        if isinstance(data, np.ndarray):
            data = np.ascontiguousarray(data)
        h = ctypes.c_void_p()
        check(lib().umapb_prebuilt_create(_dtype_code(self.dtype), data_dim, num_obs, _ptr(data), ctypes.byref(h)))
        self._h = h.value
        self.num_obs, self.data_dim = num_obs, data_dim

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                lib().umapb_prebuilt_free(self._h)
            except Exception:
                pass
            self._h = None


def initialize_prebuilt(prebuilt: Prebuilt, num_dim: int, embedding, options: Optional[Options] = None) -> Status:
    """initialize(const knncolle::Prebuilt&, num_dim, embedding, Options)
    (include/umappp/initialize.hpp:138-142) on a device-resident index."""
    options = options or Options()
    out = ctypes.c_void_p()
    copt = options.to_c()
    check(lib().umapb_initialize_prebuilt(prebuilt._h, num_dim, _ptr(embedding), ctypes.byref(copt),
                                          ctypes.byref(out)))
    return Status(out.value, prebuilt.dtype)


def initialize_from_data(data, num_dim: int, embedding, options: Optional[Options] = None,
                         num_obs: Optional[int] = None, data_dim: Optional[int] = None) -> Status:
    """initialize(data_dim, num_obs, data, builder, num_dim, embedding, Options)
    (include/umappp/initialize.hpp:165-177) with the exact device kNN as the builder.
    'data' is (num_obs, data_dim); for device pointers give num_obs and data_dim."""
    options = options or Options()
    dt = _float_dtype(data) if not isinstance(data, int) else _float_dtype(embedding)
    if num_obs is None or data_dim is None:
        shape = data.shape if isinstance(data, np.ndarray) else tuple(data.__cuda_array_interface__["shape"])
        num_obs, data_dim = int(shape[0]), int(shape[1])
    out = ctypes.c_void_p()
    copt = options.to_c()
    check(lib().umapb_initialize_data(_dtype_code(dt), data_dim, num_obs, _ptr(data), num_dim, _ptr(embedding),
                                      ctypes.byref(copt), ctypes.byref(out)))
    return Status(out.value, dt)


def knn_query(ref_data: np.ndarray, query_data: np.ndarray, k: int):
    """Exact neighbours of every query row among the reference rows
    (umapb_knn_query): (indices, distances), each (num_query, k)."""
    ref_data = np.ascontiguousarray(ref_data)
    query_data = np.ascontiguousarray(query_data, dtype=ref_data.dtype)
    nr, dim = ref_data.shape
    nq = query_data.shape[0]
    if query_data.ndim != 2 or query_data.shape[1] != dim:
        raise ValueError("query_data must have the reference data's columns")
    idx = np.zeros((nq, k), dtype=np.int32)
    dist = np.zeros((nq, k), dtype=ref_data.dtype)
    check(lib().umapb_knn_query(_dtype_code(ref_data.dtype), dim, nr, _ptr(ref_data), nq, _ptr(query_data), k,
                                _ptr(idx), _ptr(dist)))
    return idx, dist


def transform(ref_data: np.ndarray, ref_embedding: np.ndarray, new_data: np.ndarray,
              options: Optional[Options] = None, num_epochs: int = 0) -> np.ndarray:
    """Positions of new points in a finished layout (umapb_transform): their
    nearest reference points, a start at the similarity-weighted mean of those
    points' positions, then optimize_layout's steps with only the new points
    moving.  Returns (num_new, num_dim) in the reference data's type."""
    options = options or Options()
    ref_data = np.ascontiguousarray(ref_data)
    dt = ref_data.dtype
    ref_embedding = np.ascontiguousarray(ref_embedding, dtype=dt)
    new_data = np.ascontiguousarray(new_data, dtype=dt)
    nr, dim = ref_data.shape
    if ref_embedding.shape[0] != nr:
        raise ValueError("ref_embedding must have one row per reference point")
    if new_data.ndim != 2 or new_data.shape[1] != dim:
        raise ValueError("new_data must have the reference data's columns")
    num_dim = ref_embedding.shape[1]
    out = np.zeros((new_data.shape[0], num_dim), dtype=dt)
    copt = options.to_c()
    check(lib().umapb_transform(_dtype_code(dt), dim, nr, _ptr(ref_data), _ptr(ref_embedding), new_data.shape[0],
                                _ptr(new_data), num_dim, ctypes.byref(copt), int(num_epochs), _ptr(out)))
    return out


def transform_epochs(options: Optional[Options] = None, num_epochs: int = 0, num_new: int = 0) -> int:
    """The epoch count umapb_transform uses for these arguments."""
    copt = (options or Options()).to_c()
    return int(lib().umapb_transform_epochs(ctypes.byref(copt), int(num_epochs), int(num_new)))


def batch_run(data, sizes, num_dim: int, embedding, options: Optional[Options] = None) -> dict:
    """Many independent UMAP runs in one pass: instance i is the next sizes[i]
    rows of 'data' (float32/float64, (sum(sizes), data_dim)) and of 'embedding'
    ((sum(sizes), num_dim), overwritten with the final layouts).  Each instance
    gets the result of initialize_from_data + run with the same options, except
    that the optimisation draws its negative samples from a different generator
    stream.  All instances must resolve to the same epoch count (give
    num_epochs when their sizes straddle 10,000).  Returns the stage times in ms."""
    options = options or Options()
    dt = _float_dtype(data)
    sizes = np.ascontiguousarray(np.asarray(sizes, dtype=np.int32))
    shape = data.shape if isinstance(data, np.ndarray) else tuple(data.__cuda_array_interface__["shape"])
    if int(shape[0]) != int(sizes.sum()):
        raise ValueError("data must have sum(sizes) rows")
    ms = np.zeros(len(STAGES), dtype=np.float64)
    copt = options.to_c()
    check(lib().umapb_batch_run(_dtype_code(dt), len(sizes), _ptr(sizes), int(shape[1]), _ptr(data), num_dim,
                                _ptr(embedding), ctypes.byref(copt), _ptr(ms)))
    return dict(zip(STAGES, ms.tolist()))


# ------------------------------------------------------------ stage calls --

def knn_shard(data: np.ndarray, k: int, shard: int, num_shards: int):
    """One shard of knn() for a search split across ranks (umapb_knn_shard):
    (rows, indices, distances) with rows ascending and indices / distances of
    shape (len(rows), k).  The shards of 0 .. num_shards - 1 partition the rows."""
    data = np.ascontiguousarray(data)
    n, dim = data.shape
    rows = np.zeros(n, dtype=np.int32)
    idx = np.zeros((n, k), dtype=np.int32)
    dist = np.zeros((n, k), dtype=data.dtype)
    count = ctypes.c_int32()
    check(lib().umapb_knn_shard(_dtype_code(data.dtype), dim, n, _ptr(data), k, int(shard), int(num_shards),
                                _ptr(rows), _ptr(idx), _ptr(dist), ctypes.byref(count)))
    m = count.value
    return rows[:m].copy(), idx[:m].copy(), dist[:m].copy()


def knn(data: np.ndarray, k: int):
    """Exact Euclidean kNN; returns (indices int32 (n, k), distances (n, k) of data's type)."""
    n, dim = data.shape
    data = np.ascontiguousarray(data)
    idx = np.zeros((n, k), dtype=np.int32)
    dist = np.zeros((n, k), dtype=data.dtype)
    check(lib().umapb_knn(_dtype_code(data.dtype), dim, n, _ptr(data), k, _ptr(idx), _ptr(dist)))
    return idx, dist


def neighbor_similarities(neighbors, local_connectivity=1.0, bandwidth=1.0, min_k_dist_scale=1e-3,
                          use_newton=True, dtype=None, return_rho_sigma=False):
    """include/umappp/neighbor_similarities.hpp:53-207; returns the CSR triple with weights."""
    ptr, idx, val = to_csr(neighbors, dtype)
    val = val.copy()
    n = len(ptr) - 1
    rho = np.zeros(n, dtype=np.float64)
    sigma = np.zeros(n, dtype=np.float64)
    check(lib().umapb_neighbor_similarities(_dtype_code(val.dtype), n, _ptr(ptr), _ptr(val), local_connectivity,
                                            bandwidth, min_k_dist_scale, int(bool(use_newton)), _ptr(rho),
                                            _ptr(sigma)))
    if return_rho_sigma:
        return (ptr, idx, val), rho, sigma
    return ptr, idx, val


def combine_neighbor_sets(neighbors, mix_ratio=1.0, dtype=None):
    """include/umappp/combine_neighbor_sets.hpp:16-99; returns a CSR triple."""
    ptr, idx, val = to_csr(neighbors, dtype)
    n = len(ptr) - 1
    cap = max(2 * int(ptr[-1]), 1)
    optr = np.zeros(n + 1, dtype=np.int64)
    oidx = np.zeros(cap, dtype=np.int32)
    oval = np.zeros(cap, dtype=val.dtype)
    nnz = ctypes.c_int64()
    check(lib().umapb_combine_neighbor_sets(_dtype_code(val.dtype), n, _ptr(ptr), _ptr(idx), _ptr(val), mix_ratio,
                                            _ptr(optr), _ptr(oidx), _ptr(oval), cap, ctypes.byref(nnz)))
    return optr, oidx[:nnz.value].copy(), oval[:nnz.value].copy()


def similarities_to_epochs(graph, num_epochs: int, negative_sample_rate: float, dtype=None) -> EpochData:
    """include/umappp/optimize_layout.hpp:47-92."""
    ptr, idx, val = to_csr(graph, dtype)
    n = len(ptr) - 1
    cap = max(int(ptr[-1]), 1)
    optr = np.zeros(n + 1, dtype=np.int64)
    tg = np.zeros(cap, dtype=np.int32)
    arrs = [np.zeros(cap, dtype=val.dtype) for _ in range(3)]
    nnz = ctypes.c_int64()
    check(lib().umapb_similarities_to_epochs(_dtype_code(val.dtype), n, _ptr(ptr), _ptr(idx), _ptr(val), num_epochs,
                                             negative_sample_rate, _ptr(optr), _ptr(tg), *(_ptr(a) for a in arrs),
                                             ctypes.byref(nnz)))
    m = nnz.value
    return EpochData(optr, tg[:m].copy(), *(a[:m].copy() for a in arrs), total_epochs=num_epochs, current_epoch=0)


def has_multiple_components(graph) -> bool:
    """include/umappp/spectral_init.hpp:142-168."""
    ptr, idx, _ = to_csr(graph)
    out = ctypes.c_int()
    check(lib().umapb_has_multiple_components(len(ptr) - 1, _ptr(ptr), _ptr(idx), ctypes.byref(out)))
    return bool(out.value)


def spectral_init(graph, num_dim: int, embedding=None, irlba: Optional[IrlbaOptions] = None, scale=10.0,
                  jitter=False, jitter_sd=1e-4, seed=9876543210, dtype=None, return_evals=False):
    """include/umappp/spectral_init.hpp:171-207.  Returns (ok, embedding[, eigenvalues])."""
    irlba = irlba or IrlbaOptions()
    ptr, idx, val = to_csr(graph, dtype)
    n = len(ptr) - 1
    Y = np.zeros((n, num_dim), dtype=val.dtype) if embedding is None else embedding
    ok = ctypes.c_int()
    ev = np.zeros(num_dim + 1, dtype=np.float64)
    check(lib().umapb_spectral_init(_dtype_code(val.dtype), n, _ptr(ptr), _ptr(idx), _ptr(val), num_dim, _ptr(Y),
                                    irlba.extra_work, irlba.max_iterations, irlba.convergence_tolerance, scale,
                                    int(bool(jitter)), jitter_sd, seed, ctypes.byref(ok), _ptr(ev)))
    return (bool(ok.value), Y, ev) if return_evals else (bool(ok.value), Y)


def random_init(num_obs: int, num_dim: int, seed=9876543210, scale=10.0, dtype=np.float64) -> np.ndarray:
    """include/umappp/spectral_init.hpp:209-225."""
    Y = np.zeros((num_obs, num_dim), dtype=dtype)
    check(lib().umapb_random_init(_dtype_code(dtype), num_obs, num_dim, _ptr(Y), seed, scale))
    return Y


def find_ab(spread: float, min_dist: float):
    """include/umappp/find_ab.hpp:44-168."""
    a, b = ctypes.c_double(), ctypes.c_double()
    check(lib().umapb_find_ab(spread, min_dist, ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


def choose_num_epochs(num_epochs: Optional[int], num_obs: int) -> int:
    """include/umappp/initialize.hpp:27-47."""
    return lib().umapb_choose_num_epochs(0 if num_epochs is None else 1, 0 if num_epochs is None else num_epochs,
                                         num_obs)


def optimize_layout(num_dim: int, embedding: np.ndarray, epochs: EpochData, a: float, b: float, gamma: float,
                    learning_rate: float, seed: int, epoch_limit: int, negative_sample_rate: float) -> None:
    """include/umappp/optimize_layout.hpp:116-185 on the device; updates embedding and epochs in place."""
    n = len(epochs.cumulative_num_edges) - 1
    cur = ctypes.c_int(epochs.current_epoch)
    check(lib().umapb_optimize_layout(
        _dtype_code(embedding.dtype), num_dim, _ptr(embedding), n, _ptr(epochs.cumulative_num_edges),
        _ptr(epochs.edge_targets), _ptr(epochs.epochs_per_sample), _ptr(epochs.epoch_of_next_sample),
        _ptr(epochs.epoch_of_next_negative_sample), negative_sample_rate, epochs.total_epochs, ctypes.byref(cur), a,
        b, gamma, learning_rate, seed, epoch_limit))
    epochs.current_epoch = cur.value


def loss_grad(graph, embedding: np.ndarray, a: float, b: float, eps_rep: float = 0.0, with_constant: bool = False):
    """Fuzzy cross-entropy and its gradient (include/umapb.h umapb_loss_grad).
    Returns (loss, grad_embedding, (dL/da, dL/db))."""
    ptr, idx, val = to_csr(graph, embedding.dtype)
    embedding = np.ascontiguousarray(embedding)
    n, dim = embedding.shape
    g = np.zeros_like(embedding)
    gab = np.zeros(2, dtype=np.float64)
    loss = ctypes.c_double()
    check(lib().umapb_loss_grad(_dtype_code(embedding.dtype), dim, _ptr(embedding), n,
                                _ptr(ptr), _ptr(idx), _ptr(val), a, b, eps_rep, int(bool(with_constant)),
                                ctypes.byref(loss), _ptr(g), _ptr(gab)))
    return loss.value, g, (float(gab[0]), float(gab[1]))
