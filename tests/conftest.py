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
