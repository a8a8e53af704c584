"""ctypes binding of libumappp_b200.so (declarations in include/umapb.h).

The shared library is built in-tree (``python -m umappp_b200.build``) and
loaded from this directory.  There is no fallback: if the library is missing
or cannot be loaded, importing the bindings raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libumappp_b200.so")

UMAPB_OK = 0
ERR_NAMES = {1: "INVALID", 2: "OOM", 3: "CUDA", 4: "DEVICE_TIMEOUT", 5: "OVERFLOW", 6: "NO_DEVICE"}
F32, F64 = 0, 1

_c_int, _c_i32, _c_i64, _c_u64, _c_dbl, _c_size = (ctypes.c_int, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64,
                                                    ctypes.c_double, ctypes.c_size_t)
_vp = ctypes.c_void_p
_P = ctypes.POINTER


class UmapbOptions(ctypes.Structure):
    """Mirror of umapb_options (include/umapb.h)."""

    _fields_ = [
        ("local_connectivity", _c_dbl), ("bandwidth", _c_dbl), ("mix_ratio", _c_dbl), ("spread", _c_dbl),
        ("min_dist", _c_dbl), ("a", _c_dbl), ("b", _c_dbl), ("has_a", _c_int), ("has_b", _c_int),
        ("repulsion_strength", _c_dbl), ("initialize_method", _c_int),
        ("initialize_random_on_spectral_fail", _c_int), ("irlba_extra_work", _c_int),
        ("irlba_max_iterations", _c_int), ("irlba_convergence_tolerance", _c_dbl),
        ("initialize_spectral_scale", _c_dbl), ("initialize_spectral_jitter", _c_int),
        ("initialize_spectral_jitter_sd", _c_dbl), ("initialize_random_scale", _c_dbl),
        ("initialize_seed", _c_u64), ("num_epochs", _c_int), ("has_num_epochs", _c_int),
        ("learning_rate", _c_dbl), ("negative_sample_rate", _c_dbl), ("num_neighbors", _c_int),
        ("optimize_seed", _c_u64), ("num_threads", _c_int), ("num_threads_spectral", _c_int),
        ("num_threads_optimize", _c_int),
    ]


# name -> (restype, argtypes)
SIGNATURES = {
    "umapb_options_init": (None, [_P(UmapbOptions)]),
    "umapb_last_error": (ctypes.c_char_p, []),
    "umapb_version": (_c_int, []),
    "umapb_options_size": (_c_size, []),
    "umapb_launch_count": (_c_i64, []),
    "umapb_set_device_wait_limit": (_c_i64, [_c_i64]),
    "umapb_knn_query": (_c_int, [_c_int, _c_size, _c_i32, _vp, _c_i32, _vp, _c_int, _vp, _vp]),
    "umapb_transform": (_c_int, [_c_int, _c_size, _c_i32, _vp, _vp, _c_i32, _vp, _c_size, _P(UmapbOptions), _c_int, _vp]),
    "umapb_transform_epochs": (_c_int, [_P(UmapbOptions), _c_int, _c_i32]),
    "umapb_knn_shard": (_c_int, [_c_int, _c_size, _c_i32, _vp, _c_int, _c_i32, _c_i32, _vp, _vp, _vp, _P(_c_i32)]),
    "umapb_initialize_knn_matrix": (_c_int, [_c_int, _c_i32, _c_i32, _vp, _vp, _c_int, _c_size, _vp,
                                             _P(UmapbOptions), _P(_vp)]),
    "umapb_prebuilt_create": (_c_int, [_c_int, _c_size, _c_i32, _vp, _P(_vp)]),
    "umapb_prebuilt_free": (None, [_vp]),
    "umapb_initialize_prebuilt": (_c_int, [_vp, _c_size, _vp, _P(UmapbOptions), _P(_vp)]),
    "umapb_set_workspace_limit": (ctypes.c_size_t, [ctypes.c_size_t]),
    "umapb_measure_random_access": (_c_int, [_c_i64, _c_i64, _c_int, _c_int, ctypes.POINTER(_c_dbl)]),
    "umapb_initialize_neighbors": (_c_int, [_c_int, _c_i32, _vp, _vp, _vp, _c_size, _vp, _P(UmapbOptions), _P(_vp)]),
    "umapb_initialize_data": (_c_int, [_c_int, _c_size, _c_i32, _vp, _c_size, _vp, _P(UmapbOptions), _P(_vp)]),
    "umapb_status_run": (_c_int, [_vp, _vp, _c_int]),
    "umapb_status_epoch": (_c_int, [_vp]),
    "umapb_status_num_epochs": (_c_int, [_vp]),
    "umapb_status_num_observations": (_c_i32, [_vp]),
    "umapb_status_num_dimensions": (_c_size, [_vp]),
    "umapb_status_a": (_c_dbl, [_vp]),
    "umapb_status_b": (_c_dbl, [_vp]),
    "umapb_status_num_edges": (_c_i64, [_vp]),
    "umapb_status_get_epoch_data": (_c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "umapb_status_schedule_counts": (_c_int, [_vp, _c_int, _c_int, _vp]),
    "umapb_status_stage_ms": (_c_int, [_vp, _vp, _c_int]),
    "umapb_status_free": (None, [_vp]),
    "umapb_knn": (_c_int, [_c_int, _c_size, _c_i32, _vp, _c_int, _vp, _vp]),
    "umapb_knn_last_fp64_recomputed": (_c_int, []),
    "umapb_knn_last_tc_error": (_c_dbl, []),
    "umapb_knn_last_tile_pairs": (_c_i64, []),
    "umapb_knn_last_kernel_ms": (_c_dbl, []),
    "umapb_neighbor_similarities": (_c_int, [_c_int, _c_i32, _vp, _vp, _c_dbl, _c_dbl, _c_dbl, _c_int, _vp, _vp]),
    "umapb_combine_neighbor_sets": (_c_int, [_c_int, _c_i32, _vp, _vp, _vp, _c_dbl, _vp, _vp, _vp, _c_i64, _vp]),
    "umapb_similarities_to_epochs": (_c_int, [_c_int, _c_i32, _vp, _vp, _vp, _c_int, _c_dbl, _vp, _vp, _vp, _vp,
                                              _vp, _vp]),
    "umapb_has_multiple_components": (_c_int, [_c_i32, _vp, _vp, _P(_c_int)]),
    "umapb_spectral_init": (_c_int, [_c_int, _c_i32, _vp, _vp, _vp, _c_size, _vp, _c_int, _c_int, _c_dbl, _c_dbl,
                                     _c_int, _c_dbl, _c_u64, _P(_c_int), _vp]),
    "umapb_random_init": (_c_int, [_c_int, _c_i32, _c_size, _vp, _c_u64, _c_dbl]),
    "umapb_find_ab": (_c_int, [_c_dbl, _c_dbl, _P(_c_dbl), _P(_c_dbl)]),
    "umapb_choose_num_epochs": (_c_int, [_c_int, _c_int, _c_i64]),
    "umapb_optimize_layout": (_c_int, [_c_int, _c_size, _vp, _c_i32, _vp, _vp, _vp, _vp, _vp, _c_dbl, _c_int,
                                       _P(_c_int), _c_dbl, _c_dbl, _c_dbl, _c_dbl, _c_u64, _c_int]),
    "umapb_loss_grad": (_c_int, [_c_int, _c_size, _vp, _c_i32, _vp, _vp, _vp, _c_dbl, _c_dbl, _c_dbl, _c_int,
                                 _P(_c_dbl), _vp, _vp]),
    "umapb_loss_grad_noalloc": (_c_int, [_c_int, _c_size, _vp, _c_i32, _vp, _vp, _vp, _c_dbl, _c_dbl, _c_dbl, _c_int,
                                         _P(_c_dbl), _vp, _vp]),
    "umapb_batch_run": (_c_int, [_c_int, _c_i32, _vp, _c_size, _vp, _c_size, _vp, _P(UmapbOptions), _vp]),
}

_lib = None


class UmapbError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"umapb error {ERR_NAMES.get(code, code)}: {message}")
        self.code = code


def lib():
    """Loads libumappp_b200.so; raises if it is absent or fails to load."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m umappp_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        if L.umapb_options_size() != ctypes.sizeof(UmapbOptions):
            raise ImportError("umapb_options layout mismatch between the library and the binding")
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != UMAPB_OK:
        raise UmapbError(rc, lib().umapb_last_error().decode(errors="replace"))
