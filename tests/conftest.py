"""Shared fixtures: import paths, the `gpu` marker, deck factories."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "am-cfd_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.fixture(scope="session")
def lib():
    import amcfd
    return amcfd.lib()


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle_py
    oracle_py.build()
    return oracle_py.lib()


@pytest.fixture
def deckdir(tmp_path):
    return str(tmp_path)


def rel_l2(a, b):
    import numpy as np
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)
