"""Shared test setup: import paths, the `gpu` marker and golden-fixture loading.

CPU tests (-m "not gpu") check the oracle against the reference's golden
vectors, the engine's math on the host, scene generation and the C ABI's
exports.  GPU tests (-m gpu) call the engine through the C ABI and compare
with the oracle and the golden vectors.
"""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "a-differentiable-material-point-method-for-shape-morphing_b200")
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the engine through the C ABI")


from tests.helpers import load_golden  # noqa: E402


@pytest.fixture(scope="session")
def golden():
    return load_golden


@pytest.fixture(scope="session")
def gpu_ready():
    import dmpm
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without CUDA")
    dmpm.load_library()
    return True
