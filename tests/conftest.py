import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (NVIDIA B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def native_built():
    """Build the native library and the oracle once per session (no GPU needed)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_grb_build", os.path.join(ROOT, "grotor_b200", "build.py"))
    gb = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gb)
    gb.build()
    import oracle
    oracle.build()
    yield
