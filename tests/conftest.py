import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")
    config.addinivalue_line("markers", "slow: long-running parity case")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def lib():
    from multigridsoftbody_b200 import build, load
    build.build_library()
    return load()


@pytest.fixture(scope="session")
def oracle_built():
    from oracle.binding import build_oracle
    return build_oracle()


@pytest.fixture(scope="session")
def golden_cpu():
    import numpy as np
    path = os.path.join(ROOT, "tests", "golden", "ref_cpu.npz")
    return dict(np.load(path))
