"""Test configuration: the `gpu` marker (tests that need a CUDA device; run with -m gpu) and import paths for
the package (lib-magnet_b200/) and the oracle (oracle/, used here only as the checker)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
# GOLDEN holds sgd_cases.py, the option cases shared by the fixture script and the tests
for p in (ROOT, os.path.join(ROOT, "lib-magnet_b200"), GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def load(name):
        return dict(np.load(os.path.join(GOLDEN, name)))
    return load


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def mg(cuda):
    import magnet_b200
    return magnet_b200


@pytest.fixture(scope="session")
def ref():
    """the reference's compiled module (oracle/_ref), None when it was not built"""
    from oracle import oracle
    return oracle.reference()
