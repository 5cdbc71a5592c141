import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_ROOT = os.path.join(REPO, "city-scale-nlos-acoustic-engine-code_b200")
for p in (REPO, PKG_ROOT, os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """The product library, its bounds-checked twin and the oracle are built in-tree before any test."""
    from nlos_lbm import build as product_build
    import oracle

    product_build.build()
    product_build.build(check=True)
    oracle.build(ref=False)
    yield


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not _has_gpu():
        pytest.skip("no CUDA device")
    return True
