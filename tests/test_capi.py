"""The C-ABI library (CPU-side checks, no device work).

- libumappp_b200.so loads and exports every function include/umapb.h declares;
- the options defaults are the reference's (include/umappp/Options.hpp:37-218);
- host-only entry points (find_ab, choose_num_epochs) match the oracle;
- without a GPU, device entry points fail with UMAPB_ERR_NO_DEVICE instead of
  falling back to the CPU.
"""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = []
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if hdr.endswith(".h"):
            text = open(os.path.join(ROOT, "include", hdr)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"\b(umapb_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(umap):
    lib = ctypes.CDLL(umap._lib.LIB_PATH)
    names = _declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the binding covers the same set
    assert set(umap._lib.SIGNATURES) <= set(names)


def test_options_defaults(umap):
    o = umap.Options().to_c()
    assert (o.local_connectivity, o.bandwidth, o.mix_ratio, o.spread, o.min_dist) == (1, 1, 1, 1, 0.1)
    assert (o.has_a, o.has_b, o.repulsion_strength, o.initialize_method) == (0, 0, 1, 0)
    assert o.initialize_random_on_spectral_fail == 1 and o.initialize_spectral_scale == 10
    assert o.initialize_spectral_jitter == 0 and o.initialize_spectral_jitter_sd == 1e-4
    assert o.initialize_random_scale == 10 and o.initialize_seed == 9876543210
    assert o.has_num_epochs == 0 and o.learning_rate == 1 and o.negative_sample_rate == 5
    assert o.num_neighbors == 15 and o.optimize_seed == 1234567890
    assert umap._lib.lib().umapb_options_size() == ctypes.sizeof(umap._lib.UmapbOptions)


def test_host_entry_points_match_oracle(umap, oracle_mod):
    for s, m in ((1, 0.05), (1, 0.01), (2, 0.1), (200, 1), (20, 1000), (1, 0.1)):
        assert umap.find_ab(s, m) == oracle.find_ab(s, m)
    for n in (10, 1000, 10000, 10001, 20000, 10000000):
        assert umap.choose_num_epochs(None, n) == oracle.choose_num_epochs(None, n)
    assert umap.choose_num_epochs(42, 10) == 42


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="a GPU is present")
def test_no_device_fails_loudly(umap):
    with pytest.raises(umap.UmapbError) as e:
        umap.knn(np.zeros((10, 3), np.float32), 3)
    assert e.value.code == 6
    with pytest.raises(umap.UmapbError):
        umap.initialize([[(1, 1.0)], [(0, 1.0)]], 2, np.zeros((2, 2)))


def _compile_quickstart(out_path):
    import subprocess
    src = os.path.join(ROOT, "tests", "cpp", "quickstart.cpp")
    cmd = ["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), src,
           "-L" + os.path.join(ROOT, "umappp_b200"), "-lumappp_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "umappp_b200"), "-o", out_path]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_cpp_dropin_headers_compile(umap, tmp_path):
    # user code written for the reference's API compiles and links against the GPU headers
    _compile_quickstart(str(tmp_path / "quickstart"))
    assert (tmp_path / "quickstart").exists()


def test_cpp_extension_headers_compile(umap, tmp_path):
    # batch_run and loss_grad through the C++ headers: compiled and linked here, run on a GPU only
    import subprocess
    src = os.path.join(ROOT, "tests", "cpp", "extensions.cpp")
    out = str(tmp_path / "extensions")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"), src,
           "-L" + os.path.join(ROOT, "umappp_b200"), "-lumappp_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "umappp_b200"), "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert os.path.exists(out)
