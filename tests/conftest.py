"""Shared pytest setup: the `gpu` marker, repository paths, oracle build."""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(
    REPO, "machine-learning-based-implicit-physical-parametric-inference-for-cfd-simulation-promotion_b200")
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (os.path.join(REPO, "oracle"), PKG_DIR, REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle

    pyoracle.build_oracle()
    return pyoracle
