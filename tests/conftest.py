"""Shared test setup.

CPU tests (the default ``-m "not gpu"`` run) pin the oracle against known
answers and check the host-side logic; ``@pytest.mark.gpu`` tests run the CUDA
library through its C ABI and compare with the oracle bit for bit.
"""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_package():
    """The product package (directory name zkwasm-prover_b200)."""
    return importlib.import_module("zkwasm-prover_b200")


@pytest.fixture(scope="session")
def O():
    import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def zkp():
    return load_package()


@pytest.fixture(scope="session")
def gpu(zkp):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    zkp.load_library()
    return zkp
