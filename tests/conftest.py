import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cuda-pi-chudnovsky-bbp_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU; runs the CUDA path through the C ABI")


@pytest.fixture(scope="session")
def b2m_gpu():
    """The product library, initialised on device 0 (GPU tests only)."""
    import b200mul

    b200mul.init(0)
    return b200mul
