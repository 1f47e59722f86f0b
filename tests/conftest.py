"""Shared pytest fixtures.

``gpu``-marked tests need a CUDA device (they run the product's CUDA kernels
through the C ABI); everything else runs on CPU.  The oracle (oracle/, a C
restatement of the reference arithmetic) is the checker in both.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    import oracle as orc
    orc.build()
    return orc.Oracle()


@pytest.fixture(scope="session")
def reference():
    import oracle as orc
    if not orc.Reference.available():
        pytest.skip("reference build (oracle/_ref) not present")
    return orc.Reference()


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name))
    return load


@pytest.fixture(scope="session")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import parparpar_b200 as pp
    return pp.default_context(0)


@pytest.fixture
def rng():
    return np.random.default_rng(12345)
