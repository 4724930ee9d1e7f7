"""CPU checks of the C ABI library: it loads, exports every symbol the header
declares, and its host-only functions agree with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "ilc.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ilc_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(cuda_lib):
    lib = ctypes.CDLL(cuda_lib)
    names = declared_functions()
    assert len(names) >= 17
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_header(cuda_lib):
    from illcrawl_b200 import _lib
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_camera_plane_and_scale_match_oracle(cuda_lib, oracle_mod):
    import illcrawl_b200 as ilc
    rng = np.random.default_rng(3)
    for _ in range(50):
        look = rng.normal(size=3)
        look /= np.linalg.norm(look)
        args = (rng.random(3) * 1000, look, rng.random() * 6.28, 100 + rng.random() * 5000,
                int(rng.integers(16, 1025)), int(rng.integers(16, 1025)))
        a = ilc.camera_plane(ilc.camera(*args))
        b = oracle_mod.camera_setup(oracle_mod.camera(*args))
        assert np.array_equal(a, b)
        for mode in (0, 1, 2):
            lc, ac = rng.random() + 0.5, rng.random() + 0.5
            assert ilc.los_scale(ilc.camera(*args), 3000.0, lc, ac, mode) == \
                oracle_mod.los_scale(oracle_mod.camera(*args), 3000.0, lc, ac, mode)
    # look_at = z uses y as the helper axis (camera.cpp:124-136)
    p = ilc.camera_plane(ilc.camera((0, 0, 0), (0, 0, 1), 0, 10, 10, 10))
    assert np.array_equal(p[3:9], np.float32([1, 0, 0, 0, 1, 0]))


def test_create_without_device_fails_loudly(cuda_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import illcrawl_b200 as ilc
    with pytest.raises(RuntimeError):
        ilc.Context(0)


def test_gaunt_loader_matches_numpy(gaunt_table):
    t = np.loadtxt(os.path.join(ROOT, "illcrawl_b200", "data", "gaunt_factor.dat"), np.float32)
    assert np.array_equal(gaunt_table, t)
