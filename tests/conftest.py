"""Test configuration: the `gpu` marker selects tests that need an sm_100 GPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle.oracle import REFERENCE_TRUNK  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100) GPU")
    config.addinivalue_line("markers", "slow: CPU test that takes more than a few seconds")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the product library and the oracle before any test (no-op when up to date)."""
    from gpair_b200 import build as B
    B.build()
    from oracle import oracle as O
    O.build()
    yield


def reference_fixture_path():
    p = os.path.join(REFERENCE_TRUNK, "2004contest1.oifits")
    return p if os.path.exists(p) else None


def cuda_device_ok():
    try:
        import torch
        return torch.cuda.is_available() and torch.cuda.get_device_capability(0)[0] == 10
    except Exception:
        return False
