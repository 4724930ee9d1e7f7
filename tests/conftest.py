import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def cuda_lib():
    from illcrawl_b200 import build
    build.build()
    return build.LIB


@pytest.fixture(scope="session")
def gaunt_table():
    from illcrawl_b200 import load_gaunt_table
    return load_gaunt_table()


@pytest.fixture(scope="session")
def ctx(cuda_lib):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import illcrawl_b200 as ilc
    c = ilc.Context(0)
    yield c
    c.close()


def random_queries(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    q = np.zeros((n, 4), np.float32)
    q[:, :3] = (lo + rng.random((n, 3)) * (hi - lo)).astype(np.float32)
    return q


def reference_arf():
    """The reference's ARF (chandra.cpp arf_data[0:1024]) from the golden
    fixture made by tests/golden/make_golden.py: (float32 table, x_min, dx)."""
    path = os.path.join(ROOT, "tests", "golden", "chandra_arf.txt")
    x0 = dx = None
    bits = []
    for line in open(path):
        if line.startswith("#"):
            continue
        k = line.split()
        if k[0] == "x_min":
            x0 = float(k[1])
        elif k[0] == "dx":
            dx = float(k[1])
        else:
            bits.append(int(k[0], 16))
    return np.array(bits, np.uint32).view(np.float32), x0, dx
