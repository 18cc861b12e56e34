import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: large-size case")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def ref_fixture():
    import numpy as np
    return dict(np.load(os.path.join(GOLDEN, "ref_recip_23558.npz")))


@pytest.fixture(scope="session")
def fft_kat():
    import numpy as np
    return dict(np.load(os.path.join(GOLDEN, "fft_kat.npz")))


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test selected but no CUDA device is visible")
    from gpu_recip_b200 import build
    build.build()
    return torch
