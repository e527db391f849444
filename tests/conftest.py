"""Test configuration: the `gpu` marker, library/oracle fixtures.

Tests marked `gpu` need a B200 and the built CUDA library; everything else runs on
CPU (oracle pins against the reference's own code and golden fixtures, the C ABI
surface, the configuration front-end, multi-process host logic over gloo).
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the in-tree CUDA library")
    config.addinivalue_line("markers", "slow: long-running")


def _have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def have_gpu():
    return _have_gpu()


@pytest.fixture(scope="session")
def qk():
    import quantkos_b200
    return quantkos_b200


@pytest.fixture(scope="session")
def handle(qk):
    if not _have_gpu():
        pytest.skip("no CUDA device")
    h = qk.Handle(0)
    yield h
    h.close()


@pytest.fixture(scope="session")
def oracle():
    from oracle import qkoracle
    qkoracle.lib()
    return qkoracle


@pytest.fixture(scope="session")
def ref():
    from oracle import qkref
    if not qkref.available():
        pytest.skip("reference harness not built (needs the reference checkout)")
    return qkref
