"""Shared fixtures.  Markers: `gpu` = needs a CUDA device (run with -m gpu)."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_libs():
    import pyoracle
    return pyoracle.load(build=True)


@pytest.fixture(scope="session")
def orc(oracle_libs):
    return oracle_libs[0]


@pytest.fixture(scope="session")
def ref(oracle_libs):
    if oracle_libs[1] is None:
        pytest.skip("compiled reference shaders (oracle/_ref) not available")
    return oracle_libs[1]


@pytest.fixture(scope="session")
def product():
    from retrocam_b200 import build, api
    build.build()
    api.lib()
    return api


@pytest.fixture(scope="session")
def cuda_ok(product):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return True


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a
