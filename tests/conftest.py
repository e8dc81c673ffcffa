import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "fideslib-fork_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run on the B200 box)")


@pytest.fixture(scope="session", autouse=True)
def _built_oracle():
    import oracle
    oracle.build()
    yield


@pytest.fixture(scope="session")
def fides():
    """The GPU library.  Builds it when absent; never falls back to anything else."""
    import torch
    import fides_b200
    fides_b200.build()
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without a CUDA device")
    return fides_b200
