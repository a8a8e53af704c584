"""Oracle: CPU checkers for the UMAP hot path (test infrastructure only).

Two checkers live here, neither of which is ever part of the product path:

* ``liboracle.so`` -- a plain-C restatement of the reference's stages
  (``oracle.c``/``oracle_impl.h``, each function citing the reference file and
  lines it follows), plus an exact FP64 brute-force kNN, trustworthiness and
  the fuzzy cross-entropy with its gradient.
* ``_ref/libumappp_ref.so`` -- the reference's own headers (libscran/umappp
  v3.3.2, ``include/umappp/*.hpp``) compiled unmodified against project-written
  stand-ins for its absent dependencies (``ref_shim/``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  Arrays follow the reference's layout:
observation ``i`` of a data or embedding matrix occupies
``[i * dim, (i + 1) * dim)``; neighbour lists and graphs are CSR with int64
row pointers and int32 indices.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libumappp_ref.so")

_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_c_int = ctypes.c_int
_c_i64 = ctypes.c_int64
_c_u64 = ctypes.c_uint64
_c_dbl = ctypes.c_double
_vp = ctypes.c_void_p

_lib = None
_ref = None


def build() -> None:
    """Compile liboracle.so, and _ref from the reference's headers when its
    source tree is present ($UMAPB_REFERENCE, else /root/reference)."""
    ref = os.environ.get("UMAPB_REFERENCE", "/root/reference")
    args = ["make", "-s", "-C", HERE]
    if os.path.isdir(os.path.join(ref, "include", "umappp")):
        args.append(f"REFERENCE={ref}")
    subprocess.run(args, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        for suf, fp in (("f64", _f64p), ("f32", _f32p)):
            getattr(L, f"oracle_neighbor_similarities_{suf}").argtypes = [
                _c_int, _i64p, fp, _c_dbl, _c_dbl, _c_dbl, _c_int, fp, fp]
            f = getattr(L, f"oracle_combine_neighbor_sets_{suf}")
            f.argtypes = [_c_int, _i64p, _i32p, fp, _c_dbl, _i64p, _i32p, fp]
            f.restype = _c_i64
            f = getattr(L, f"oracle_similarities_to_epochs_{suf}")
            f.argtypes = [_c_int, _i64p, _i32p, fp, _c_int, _c_dbl, _i64p, _i32p, fp, fp, fp]
            f.restype = _c_i64
            getattr(L, f"oracle_random_init_{suf}").argtypes = [_c_int, _c_int, fp, _c_u64, _c_dbl]
            getattr(L, f"oracle_optimize_layout_{suf}").argtypes = [
                _c_int, fp, _c_int, _i64p, _i32p, fp, fp, fp, _c_dbl, _c_int, ctypes.POINTER(_c_int),
                _c_dbl, _c_dbl, _c_dbl, _c_dbl, _c_u64, _c_int, _vp]
            getattr(L, f"oracle_transform_layout_{suf}").argtypes = [
                _c_int, fp, _c_int, _i64p, _i32p, fp, fp, fp, _c_dbl, _c_int, fp, _c_int, _c_int,
                _c_dbl, _c_dbl, _c_dbl, _c_dbl, _c_u64]
            getattr(L, f"oracle_has_multiple_components_{suf}").argtypes = [_c_int, _i64p, _i32p]
            f = getattr(L, f"oracle_spectral_init_{suf}")
            f.argtypes = [_c_int, _i64p, _i32p, fp, _c_int, fp, _c_int, _c_int, _c_dbl, _c_dbl, _c_int, _c_dbl,
                          _c_u64, _vp]
            f.restype = _c_int
        L.oracle_find_ab.argtypes = [_c_dbl, _c_dbl, ctypes.POINTER(_c_dbl), ctypes.POINTER(_c_dbl)]
        L.oracle_choose_num_epochs.argtypes = [_c_int, _c_int, _c_i64]
        L.oracle_choose_num_epochs.restype = _c_int
        L.oracle_mt64_stream.argtypes = [_c_u64, _c_i64, _u64p]
        L.oracle_knn_f64.argtypes = [_c_int, _c_int, _f64p, _c_int, _c_int, _c_int, _i32p, _f64p]
        L.oracle_knn_f32.argtypes = [_c_int, _c_int, _f32p, _c_int, _c_int, _c_int, _i32p, _f64p]
        L.oracle_knn_query_f64.argtypes = [_c_int, _c_int, _c_int, _f64p, _f64p, _c_int, _i32p, _f64p]
        L.oracle_negstream_draws.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _c_u64,
                                             ctypes.c_uint32, _c_int, _i32p]
        L.oracle_trustworthiness.argtypes = [_c_int, _c_int, _f64p, _c_int, _f64p, _c_int, _c_int, _i32p]
        L.oracle_trustworthiness.restype = _c_dbl
        L.oracle_cross_entropy.argtypes = [_c_int, _i64p, _i32p, _f64p, _c_int, _f64p, _c_dbl, _c_dbl]
        L.oracle_cross_entropy.restype = _c_dbl
        L.oracle_loss_grad.argtypes = [_c_int, _i64p, _i32p, _f64p, _c_int, _f64p, _c_dbl, _c_dbl, _c_dbl, _f64p, _f64p]
        L.oracle_loss_grad.restype = _c_dbl
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref():
    """The reference's headers compiled against the stand-ins (oracle/_ref)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_PATH):
            raise FileNotFoundError(f"{REF_PATH} is not built (it needs the reference sources)")
        R = ctypes.CDLL(REF_PATH)
        R.ref_last_error.restype = ctypes.c_char_p
        R.ref_choose_num_epochs.argtypes = [_c_int, _c_int, _c_int]
        R.ref_find_ab.argtypes = [_c_dbl, _c_dbl, ctypes.POINTER(_c_dbl), ctypes.POINTER(_c_dbl)]
        for suf, fp in (("f64", _f64p), ("f32", _f32p)):
            getattr(R, f"ref_neighbor_similarities_{suf}").argtypes = [
                _c_int, _i64p, _i32p, fp, _c_dbl, _c_dbl, _c_dbl, _c_int, _c_int]
            f = getattr(R, f"ref_combine_neighbor_sets_{suf}")
            f.argtypes = [_c_int, _i64p, _i32p, fp, _c_dbl, _i64p, _i32p, fp, _c_i64]
            f.restype = _c_i64
            f = getattr(R, f"ref_similarities_to_epochs_{suf}")
            f.argtypes = [_c_int, _i64p, _i32p, fp, _c_int, _c_dbl, _i64p, _i32p, fp, fp, fp]
            f.restype = _c_i64
            getattr(R, f"ref_spectral_init_{suf}").argtypes = [
                _c_int, _i64p, _i32p, fp, _c_int, fp, _c_dbl, _c_int, _c_dbl, _c_int, _c_dbl, _c_u64, _c_int]
            getattr(R, f"ref_random_init_{suf}").argtypes = [_c_int, _c_int, fp, _c_u64, _c_dbl]
            getattr(R, f"ref_has_multiple_components_{suf}").argtypes = [_c_int, _i64p, _i32p, fp]
            getattr(R, f"ref_optimize_layout_{suf}").argtypes = [
                _c_int, fp, _c_int, _i64p, _i32p, fp, fp, fp, _c_dbl, _c_int, ctypes.POINTER(_c_int),
                _c_dbl, _c_dbl, _c_dbl, _c_dbl, _c_u64, _c_int, _c_int]
            getattr(R, f"ref_knn_{suf}").argtypes = [_c_int, _c_int, fp, _c_int, _c_int, _c_int, _c_int, _i32p, fp]
            for name in ("ref_status_from_neighbors", "ref_status_from_data"):
                getattr(R, f"{name}_{suf}").restype = _vp
            getattr(R, f"ref_status_from_neighbors_{suf}").argtypes = [_c_int, _i64p, _i32p, fp, _c_int, fp, _vp]
            getattr(R, f"ref_status_from_data_{suf}").argtypes = [_c_int, _c_int, fp, _c_int, fp, _vp]
            getattr(R, f"ref_status_run_{suf}").argtypes = [_vp, fp, _c_int]
            getattr(R, f"ref_status_epoch_{suf}").argtypes = [_vp]
            getattr(R, f"ref_status_num_epochs_{suf}").argtypes = [_vp]
            getattr(R, f"ref_status_num_edges_{suf}").argtypes = [_vp]
            getattr(R, f"ref_status_num_edges_{suf}").restype = _c_i64
            getattr(R, f"ref_status_epoch_data_{suf}").argtypes = [_vp, _i64p, _i32p, fp, fp, fp]
            getattr(R, f"ref_status_destroy_{suf}").argtypes = [_vp]
        _ref = R
    return _ref


def _suf(dtype) -> str:
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


def _check(rc, R=None):
    if rc < 0:
        msg = (R or ref()).ref_last_error().decode()
        raise RuntimeError(msg)
    return rc


# --------------------------------------------------------------------------
# Data containers


@dataclass
class CSR:
    """Row-compressed neighbour list or graph: row i is idx/val[ptr[i]:ptr[i+1]]."""

    ptr: np.ndarray
    idx: np.ndarray
    val: np.ndarray

    @property
    def n(self) -> int:
        return len(self.ptr) - 1

    @property
    def nnz(self) -> int:
        return int(self.ptr[-1])

    def copy(self) -> "CSR":
        return CSR(self.ptr.copy(), self.idx.copy(), self.val.copy())

    def astype(self, dtype) -> "CSR":
        return CSR(self.ptr, self.idx, np.ascontiguousarray(self.val, dtype=dtype))

    @staticmethod
    def from_dense(idx: np.ndarray, val: np.ndarray) -> "CSR":
        n, k = idx.shape
        ptr = np.arange(n + 1, dtype=np.int64) * k
        return CSR(ptr, np.ascontiguousarray(idx.reshape(-1), dtype=np.int32), np.ascontiguousarray(val.reshape(-1)))

    @staticmethod
    def from_lists(rows, dtype=np.float64) -> "CSR":
        ptr = np.zeros(len(rows) + 1, dtype=np.int64)
        for i, r in enumerate(rows):
            ptr[i + 1] = ptr[i] + len(r)
        idx = np.array([j for r in rows for j, _ in r], dtype=np.int32)
        val = np.array([v for r in rows for _, v in r], dtype=dtype)
        return CSR(ptr, idx, val)

    def to_lists(self):
        return [list(zip(self.idx[self.ptr[i]:self.ptr[i + 1]].tolist(), self.val[self.ptr[i]:self.ptr[i + 1]].tolist()))
                for i in range(self.n)]


@dataclass
class EpochData:
    """The reference's EpochData (include/umappp/optimize_layout.hpp:27-45) as arrays."""

    ptr: np.ndarray
    targets: np.ndarray
    eps: np.ndarray
    enext: np.ndarray
    enneg: np.ndarray
    total_epochs: int
    rate: float
    current_epoch: int = 0

    def copy(self) -> "EpochData":
        return EpochData(self.ptr.copy(), self.targets.copy(), self.eps.copy(), self.enext.copy(), self.enneg.copy(),
                         self.total_epochs, self.rate, self.current_epoch)


# --------------------------------------------------------------------------
# The C restatement


def mt64_stream(seed: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint64)
    lib().oracle_mt64_stream(seed, count, out)
    return out


def knn(data: np.ndarray, k: int, qstart: int = 0, qcount: int | None = None):
    """Exact FP64 kNN; data is (n, dim).  Returns (idx int32 (q, k), dist float64 (q, k))."""
    n, dim = data.shape
    qcount = n - qstart if qcount is None else qcount
    idx = np.zeros((qcount, k), dtype=np.int32)
    dist = np.zeros((qcount, k), dtype=np.float64)
    if data.dtype == np.float64:
        lib().oracle_knn_f64(n, dim, np.ascontiguousarray(data), k, qstart, qcount, idx.reshape(-1), dist.reshape(-1))
    else:
        lib().oracle_knn_f32(n, dim, np.ascontiguousarray(data, dtype=np.float32), k, qstart, qcount,
                             idx.reshape(-1), dist.reshape(-1))
    return idx, dist


def neighbor_similarities(nl: CSR, local_connectivity=1.0, bandwidth=1.0, min_k_dist_scale=1e-3, use_newton=True):
    """Returns (weights CSR, rho, sigma); rows with an early return have NaN rho/sigma."""
    out = nl.copy()
    suf = _suf(out.val.dtype)
    rho = np.zeros(nl.n, dtype=out.val.dtype)
    sigma = np.zeros(nl.n, dtype=out.val.dtype)
    getattr(lib(), f"oracle_neighbor_similarities_{suf}")(nl.n, out.ptr, out.val, local_connectivity, bandwidth,
                                                           min_k_dist_scale, int(use_newton), rho, sigma)
    return out, rho, sigma


def combine_neighbor_sets(nl: CSR, mix_ratio=1.0) -> CSR:
    suf = _suf(nl.val.dtype)
    cap = max(2 * nl.nnz, 1)
    ptr = np.zeros(nl.n + 1, dtype=np.int64)
    idx = np.zeros(cap, dtype=np.int32)
    val = np.zeros(cap, dtype=nl.val.dtype)
    nnz = getattr(lib(), f"oracle_combine_neighbor_sets_{suf}")(nl.n, nl.ptr, nl.idx, nl.val, mix_ratio, ptr, idx, val)
    return CSR(ptr, idx[:nnz].copy(), val[:nnz].copy())


def similarities_to_epochs(g: CSR, num_epochs: int, rate: float) -> EpochData:
    suf = _suf(g.val.dtype)
    cap = max(g.nnz, 1)
    ptr = np.zeros(g.n + 1, dtype=np.int64)
    targets = np.zeros(cap, dtype=np.int32)
    arrs = [np.zeros(cap, dtype=g.val.dtype) for _ in range(3)]
    nnz = getattr(lib(), f"oracle_similarities_to_epochs_{suf}")(g.n, g.ptr, g.idx, g.val, num_epochs, rate, ptr,
                                                                  targets, *arrs)
    return EpochData(ptr, targets[:nnz].copy(), *(a[:nnz].copy() for a in arrs), total_epochs=num_epochs, rate=rate)


def optimize_layout(num_dim: int, embedding: np.ndarray, ep: EpochData, a: float, b: float, gamma: float,
                    alpha: float, seed: int, epoch_limit: int, counts: bool = False):
    """Serial SGD in place on (embedding, ep).  With counts=True returns an
    (epochs, 2) array of [firing edges, negative samples drawn] per epoch."""
    suf = _suf(embedding.dtype)
    cur = ctypes.c_int(ep.current_epoch)
    nep = max(epoch_limit - ep.current_epoch, 0)
    cnt = np.zeros((max(nep, 1), 2), dtype=np.int64)
    n = len(ep.ptr) - 1
    getattr(lib(), f"oracle_optimize_layout_{suf}")(
        num_dim, embedding.reshape(-1), n, ep.ptr, ep.targets, ep.eps, ep.enext, ep.enneg, ep.rate,
        ep.total_epochs, ctypes.byref(cur), a, b, gamma, alpha, seed, epoch_limit,
        cnt.ctypes.data_as(ctypes.c_void_p) if counts else None)
    ep.current_epoch = cur.value
    return cnt[:nep] if counts else None


def find_ab(spread: float, min_dist: float):
    a, b = ctypes.c_double(), ctypes.c_double()
    lib().oracle_find_ab(spread, min_dist, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def choose_num_epochs(num_epochs, n: int) -> int:
    return lib().oracle_choose_num_epochs(0 if num_epochs is None else 1, 0 if num_epochs is None else num_epochs, n)


def has_multiple_components(g: CSR) -> bool:
    return bool(getattr(lib(), f"oracle_has_multiple_components_{_suf(g.val.dtype)}")(g.n, g.ptr, g.idx))


def spectral_init(g: CSR, num_dim: int, scale=10.0, tol=1e-6, max_restarts=1000, ncv=0, jitter=False,
                  jitter_sd=1e-4, seed=9876543210, Y: np.ndarray | None = None):
    """Returns (ok, Y (n, num_dim), eigenvalues of I + D^-1/2 W D^-1/2 (num_dim + 1))."""
    dt = g.val.dtype
    Y = np.zeros((g.n, num_dim), dtype=dt) if Y is None else Y
    ev = np.zeros(num_dim + 1, dtype=np.float64)
    ok = getattr(lib(), f"oracle_spectral_init_{_suf(dt)}")(
        g.n, g.ptr, g.idx, g.val, num_dim, Y.reshape(-1), ncv, max_restarts, tol, scale, int(jitter), jitter_sd, seed,
        ev.ctypes.data_as(ctypes.c_void_p))
    return bool(ok), Y, ev


def random_init(n: int, num_dim: int, seed=9876543210, scale=10.0, dtype=np.float64) -> np.ndarray:
    out = np.zeros((n, num_dim), dtype=dtype)
    getattr(lib(), f"oracle_random_init_{_suf(dtype)}")(n, num_dim, out.reshape(-1), seed, scale)
    return out


def trustworthiness(X: np.ndarray, Y: np.ndarray, k: int = 15, queries: np.ndarray | None = None) -> float:
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    n = X.shape[0]
    q = np.arange(n, dtype=np.int32) if queries is None else np.ascontiguousarray(queries, dtype=np.int32)
    return lib().oracle_trustworthiness(n, X.shape[1], X.reshape(-1), Y.shape[1], Y.reshape(-1), k, len(q), q)


def cross_entropy(g: CSR, Y: np.ndarray, a: float, b: float) -> float:
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    return lib().oracle_cross_entropy(g.n, g.ptr, g.idx, np.ascontiguousarray(g.val, dtype=np.float64),
                                      Y.shape[1], Y.reshape(-1), a, b)


def loss_grad(g: CSR, Y: np.ndarray, a: float, b: float, eps_rep: float = 0.0):
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    gY = np.zeros_like(Y)
    gab = np.zeros(2, dtype=np.float64)
    loss = lib().oracle_loss_grad(g.n, g.ptr, g.idx, np.ascontiguousarray(g.val, dtype=np.float64), Y.shape[1],
                                  Y.reshape(-1), a, b, eps_rep, gY.reshape(-1), gab)
    return loss, gY, gab


# --------------------------------------------------------------------------
# The reference compiled from its headers (oracle/_ref)


class RefOptions(ctypes.Structure):
    """Mirror of RefOptions in ref_capi.cpp (the reference's Options, include/umappp/Options.hpp:37-218)."""

    _fields_ = [
        ("local_connectivity", ctypes.c_double), ("bandwidth", ctypes.c_double), ("mix_ratio", ctypes.c_double),
        ("spread", ctypes.c_double), ("min_dist", ctypes.c_double), ("a", ctypes.c_double), ("b", ctypes.c_double),
        ("has_a", ctypes.c_int), ("has_b", ctypes.c_int), ("repulsion_strength", ctypes.c_double),
        ("initialize_method", ctypes.c_int), ("initialize_random_on_spectral_fail", ctypes.c_int),
        ("irlba_extra_work", ctypes.c_int), ("irlba_max_iterations", ctypes.c_int),
        ("irlba_convergence_tolerance", ctypes.c_double), ("initialize_spectral_scale", ctypes.c_double),
        ("initialize_spectral_jitter", ctypes.c_int), ("initialize_spectral_jitter_sd", ctypes.c_double),
        ("initialize_random_scale", ctypes.c_double), ("initialize_seed", ctypes.c_uint64),
        ("num_epochs", ctypes.c_int), ("has_num_epochs", ctypes.c_int), ("learning_rate", ctypes.c_double),
        ("negative_sample_rate", ctypes.c_double), ("num_neighbors", ctypes.c_int),
        ("optimize_seed", ctypes.c_uint64), ("num_threads", ctypes.c_int), ("num_threads_spectral", ctypes.c_int),
        ("num_threads_optimize", ctypes.c_int),
    ]

    @staticmethod
    def defaults(**kw) -> "RefOptions":
        o = RefOptions(local_connectivity=1, bandwidth=1, mix_ratio=1, spread=1, min_dist=0.1, a=0, b=0, has_a=0,
                       has_b=0, repulsion_strength=1, initialize_method=0, initialize_random_on_spectral_fail=1,
                       irlba_extra_work=7, irlba_max_iterations=1000, irlba_convergence_tolerance=1e-6,
                       initialize_spectral_scale=10, initialize_spectral_jitter=0, initialize_spectral_jitter_sd=1e-4,
                       initialize_random_scale=10, initialize_seed=9876543210, num_epochs=0, has_num_epochs=0,
                       learning_rate=1, negative_sample_rate=5, num_neighbors=15, optimize_seed=1234567890,
                       num_threads=1, num_threads_spectral=1, num_threads_optimize=1)
        for key, value in kw.items():
            if key == "num_epochs" and value is not None:
                o.num_epochs, o.has_num_epochs = value, 1
            elif key == "a" and value is not None:
                o.a, o.has_a = value, 1
            elif key == "b" and value is not None:
                o.b, o.has_b = value, 1
            else:
                setattr(o, key, value)
        return o


class RefStatus:
    """The reference's Status (include/umappp/Status.hpp:25-141) behind ctypes."""

    def __init__(self, handle, suf):
        self.h = handle
        self.suf = suf

    def run(self, embedding: np.ndarray, epoch_limit: int | None = None):
        limit = self.num_epochs() if epoch_limit is None else epoch_limit
        _check(getattr(ref(), f"ref_status_run_{self.suf}")(self.h, embedding.reshape(-1), limit))

    def epoch(self) -> int:
        return getattr(ref(), f"ref_status_epoch_{self.suf}")(self.h)

    def num_epochs(self) -> int:
        return getattr(ref(), f"ref_status_num_epochs_{self.suf}")(self.h)

    def epoch_data(self, n: int) -> EpochData:
        R = ref()
        nnz = getattr(R, f"ref_status_num_edges_{self.suf}")(self.h)
        dt = np.float64 if self.suf == "f64" else np.float32
        ptr = np.zeros(n + 1, dtype=np.int64)
        targets = np.zeros(max(nnz, 1), dtype=np.int32)
        arrs = [np.zeros(max(nnz, 1), dtype=dt) for _ in range(3)]
        getattr(R, f"ref_status_epoch_data_{self.suf}")(self.h, ptr, targets, *arrs)
        return EpochData(ptr, targets[:nnz], *(a[:nnz] for a in arrs), total_epochs=self.num_epochs(), rate=0.0,
                         current_epoch=self.epoch())

    def __del__(self):
        if getattr(self, "h", None):
            getattr(ref(), f"ref_status_destroy_{self.suf}")(self.h)
            self.h = None


def ref_initialize(nl: CSR, num_dim: int, embedding: np.ndarray, **options) -> RefStatus:
    suf = _suf(nl.val.dtype)
    opts = RefOptions.defaults(**options)
    h = getattr(ref(), f"ref_status_from_neighbors_{suf}")(nl.n, nl.ptr, nl.idx, nl.val, num_dim, embedding.reshape(-1),
                                                            ctypes.byref(opts))
    if not h:
        raise RuntimeError(ref().ref_last_error().decode())
    return RefStatus(h, suf)


def ref_initialize_from_data(data: np.ndarray, num_dim: int, embedding: np.ndarray, **options) -> RefStatus:
    suf = _suf(data.dtype)
    opts = RefOptions.defaults(**options)
    n, dim = data.shape
    h = getattr(ref(), f"ref_status_from_data_{suf}")(dim, n, np.ascontiguousarray(data).reshape(-1), num_dim,
                                                       embedding.reshape(-1), ctypes.byref(opts))
    if not h:
        raise RuntimeError(ref().ref_last_error().decode())
    return RefStatus(h, suf)


def ref_knn(data: np.ndarray, k: int, qstart: int = 0, qcount: int | None = None, nthreads: int = 1):
    n, dim = data.shape
    qcount = n - qstart if qcount is None else qcount
    idx = np.zeros((qcount, k), dtype=np.int32)
    dist = np.zeros((qcount, k), dtype=data.dtype)
    _check(getattr(ref(), f"ref_knn_{_suf(data.dtype)}")(dim, n, np.ascontiguousarray(data).reshape(-1), k, qstart,
                                                          qcount, nthreads, idx.reshape(-1), dist.reshape(-1)))
    return idx, dist


def ref_neighbor_similarities(nl: CSR, local_connectivity=1.0, bandwidth=1.0, min_k_dist_scale=1e-3, use_newton=True,
                              num_threads=1) -> CSR:
    out = nl.copy()
    _check(getattr(ref(), f"ref_neighbor_similarities_{_suf(out.val.dtype)}")(
        nl.n, out.ptr, out.idx, out.val, local_connectivity, bandwidth, min_k_dist_scale, int(use_newton), num_threads))
    return out


def ref_combine_neighbor_sets(nl: CSR, mix_ratio=1.0) -> CSR:
    cap = max(2 * nl.nnz, 1)
    ptr = np.zeros(nl.n + 1, dtype=np.int64)
    idx = np.zeros(cap, dtype=np.int32)
    val = np.zeros(cap, dtype=nl.val.dtype)
    nnz = _check(getattr(ref(), f"ref_combine_neighbor_sets_{_suf(nl.val.dtype)}")(
        nl.n, nl.ptr, nl.idx, nl.val, mix_ratio, ptr, idx, val, cap))
    return CSR(ptr, idx[:nnz].copy(), val[:nnz].copy())


def ref_similarities_to_epochs(g: CSR, num_epochs: int, rate: float) -> EpochData:
    cap = max(g.nnz, 1)
    ptr = np.zeros(g.n + 1, dtype=np.int64)
    targets = np.zeros(cap, dtype=np.int32)
    arrs = [np.zeros(cap, dtype=g.val.dtype) for _ in range(3)]
    nnz = _check(getattr(ref(), f"ref_similarities_to_epochs_{_suf(g.val.dtype)}")(
        g.n, g.ptr, g.idx, g.val, num_epochs, rate, ptr, targets, *arrs))
    return EpochData(ptr, targets[:nnz].copy(), *(a[:nnz].copy() for a in arrs), total_epochs=num_epochs, rate=rate)


def ref_optimize_layout(num_dim: int, embedding: np.ndarray, ep: EpochData, a: float, b: float, gamma: float,
                        alpha: float, seed: int, epoch_limit: int, nthreads: int = 1):
    cur = ctypes.c_int(ep.current_epoch)
    n = len(ep.ptr) - 1
    _check(getattr(ref(), f"ref_optimize_layout_{_suf(embedding.dtype)}")(
        num_dim, embedding.reshape(-1), n, ep.ptr, ep.targets, ep.eps, ep.enext, ep.enneg, ep.rate, ep.total_epochs,
        ctypes.byref(cur), a, b, gamma, alpha, seed, epoch_limit, nthreads))
    ep.current_epoch = cur.value


def ref_find_ab(spread: float, min_dist: float):
    a, b = ctypes.c_double(), ctypes.c_double()
    _check(ref().ref_find_ab(spread, min_dist, ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


def ref_spectral_init(g: CSR, num_dim: int, scale=10.0, tol=1e-6, max_iter=1000, jitter=False, jitter_sd=1e-4,
                      seed=9876543210, nthreads=1, Y=None):
    Y = np.zeros((g.n, num_dim), dtype=g.val.dtype) if Y is None else Y
    ok = _check(getattr(ref(), f"ref_spectral_init_{_suf(g.val.dtype)}")(
        g.n, g.ptr, g.idx, g.val, num_dim, Y.reshape(-1), tol, max_iter, scale, int(jitter), jitter_sd, seed, nthreads))
    return bool(ok), Y


def ref_random_init(n: int, num_dim: int, seed=9876543210, scale=10.0, dtype=np.float64) -> np.ndarray:
    out = np.zeros((n, num_dim), dtype=dtype)
    _check(getattr(ref(), f"ref_random_init_{_suf(dtype)}")(n, num_dim, out.reshape(-1), seed, scale))
    return out


def ref_has_multiple_components(g: CSR) -> bool:
    return bool(_check(getattr(ref(), f"ref_has_multiple_components_{_suf(g.val.dtype)}")(g.n, g.ptr, g.idx, g.val)))


# --------------------------------------------------------------------------
# Seeded synthetic inputs


def gaussian_mixture(n: int, dim: int, n_clusters: int, centre_sd: float, seed: int, weights: str = "equal",
                     dtype=np.float32) -> np.ndarray:
    """Points = centre + N(0, I); centres ~ N(0, centre_sd^2 I); cluster weights
    equal or Dirichlet(1).  Returns an (n, dim) array."""
    rng = np.random.default_rng(seed)
    centres = rng.normal(0.0, centre_sd, size=(n_clusters, dim))
    if weights == "dirichlet":
        p = rng.dirichlet(np.ones(n_clusters))
    else:
        p = np.full(n_clusters, 1.0 / n_clusters)
    labels = rng.choice(n_clusters, size=n, p=p)
    pts = centres[labels] + rng.normal(0.0, 1.0, size=(n, dim))
    return np.ascontiguousarray(pts, dtype=dtype)


def knn_query(ref: np.ndarray, queries: np.ndarray, k: int):
    """Exact FP64 neighbours of every query row among the reference rows:
    (idx int32 (nq, k), dist float64 (nq, k)), ties by index."""
    ref64 = np.ascontiguousarray(ref, dtype=np.float64)
    q64 = np.ascontiguousarray(queries, dtype=np.float64)
    nq = q64.shape[0]
    idx = np.zeros((nq, k), dtype=np.int32)
    dist = np.zeros((nq, k), dtype=np.float64)
    lib().oracle_knn_query_f64(ref64.shape[0], nq, ref64.shape[1], ref64, q64, k, idx.reshape(-1), dist.reshape(-1))
    return idx, dist


def negstream_draws(head: int, tail: int, epoch: int, seed: int, n: int, count: int) -> np.ndarray:
    """'count' bounded draws in [0, n) of the negative-sample stream of one edge."""
    out = np.zeros(count, dtype=np.int32)
    lib().oracle_negstream_draws(head, tail, epoch, seed, n, count, out)
    return out


def transform_epochs(num_epochs: int, has_layout_epochs: bool, layout_epochs: int, num_new: int) -> int:
    """Epoch count of a transform: the given count, else a third of the
    layout's when set, else 100 up to 10,000 new points and 30 above."""
    if num_epochs > 0:
        return num_epochs
    if has_layout_epochs and layout_epochs > 0:
        return max(1, layout_epochs // 3)
    return 100 if num_new <= 10000 else 30


def transform(ref_data: np.ndarray, ref_embedding: np.ndarray, new_data: np.ndarray, k: int, num_epochs: int,
              a: float, b: float, gamma: float = 1.0, learning_rate: float = 1.0, negative_sample_rate: float = 5.0,
              seed: int = 1234567890, local_connectivity: float = 1.0, bandwidth: float = 1.0):
    """The transform of new points into a finished layout, serially (the
    device's umapb_transform): exact FP64 neighbours among the reference
    points, their similarities, a start at the similarity-weighted mean of the
    neighbours' positions (FP64 sums in edge order), the schedule of
    similarities_to_epochs and the head-only steps of oracle_transform_layout
    at a quarter of the learning rate.  Float type of ref_embedding.
    Returns (embedding, init, idx, weights)."""
    dt = np.asarray(ref_embedding).dtype
    suf = _suf(dt)
    nref = ref_data.shape[0]
    nq = new_data.shape[0]
    idx, dist = knn_query(ref_data, new_data, k)
    nl = CSR(np.arange(0, (nq + 1) * k, k, dtype=np.int64), idx.reshape(-1).copy(),
             dist.reshape(-1).astype(dt))
    w, _, _ = neighbor_similarities(nl, local_connectivity, bandwidth)
    yref = np.ascontiguousarray(ref_embedding, dtype=dt)
    num_dim = yref.shape[1]
    wv = w.val.astype(np.float64).reshape(nq, k)
    init = np.zeros((nq, num_dim), dtype=np.float64)
    for i in range(nq):
        ws = 0.0
        for j in range(k):
            ws += wv[i, j]
        for d in range(num_dim):
            acc = 0.0
            for j in range(k):
                acc += (wv[i, j] if ws > 0 else 1.0) * float(yref[idx[i, j], d])
            init[i, d] = acc / (ws if ws > 0 else k)
    init = init.astype(dt)
    ep = similarities_to_epochs(w, num_epochs, negative_sample_rate)
    Y = init.copy()
    getattr(lib(), f"oracle_transform_layout_{suf}")(
        num_dim, Y.reshape(-1), nq, ep.ptr, ep.targets, ep.eps, ep.enext, ep.enneg, ep.rate, num_epochs,
        yref.reshape(-1), nref, nref, a, b, gamma, learning_rate / 4.0, seed)
    return Y, init, idx, w
