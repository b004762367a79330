"""Test configuration: the `gpu` marker and shared fixtures.

`pytest -m "not gpu"` runs on any machine (oracle against the reference's
golden vectors, host-side logic, the C ABI's exported symbols). `pytest -m gpu`
needs a B200: it runs the CUDA library through its C ABI against the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Builds the oracle and the CUDA library if their shared objects are missing."""
    import oracle
    oracle.lib()
    from cindergs_b200 import _abi, build
    if not os.path.exists(_abi.LIB_PATH):
        build.build()
    yield


@pytest.fixture(scope="session")
def gpu_state():
    from cindergs_b200 import GpuPipelineState
    st = GpuPipelineState(0)
    yield st
    st.close()
