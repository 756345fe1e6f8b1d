import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a library)")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def ntcfd_lib():
    from ntustcfdlab_b200 import abi, build
    build.build()
    return abi.load_library()


@pytest.fixture(scope="session")
def orc():
    from oracle import cpu_oracle
    cpu_oracle.build()
    return cpu_oracle


def interior(a: np.ndarray) -> np.ndarray:
    """Interior 1..n of a halo array stored with index i+2."""
    return a[2:-2, 2:-2, 2:-2]


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    nb = float(np.linalg.norm(b))
    d = float(np.linalg.norm(a - b))
    return d / nb if nb > 0 else d
