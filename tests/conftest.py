import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    """The C restatement of the reference path (built on demand)."""
    from oracle import oracle as orc
    if not os.path.exists(orc.ORACLE_SO):
        orc.build()
    return orc.Oracle()


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return {name[:-4]: dict(np.load(os.path.join(GOLDEN, name)))
            for name in os.listdir(GOLDEN) if name.endswith(".npz")}


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu-marked test run without a CUDA device")
    return torch.device("cuda:0")
