import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libufem_gpu.so")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    """Build the oracle restatement once per session (plain gcc, seconds)."""
    import subprocess
    so = os.path.join(ROOT, "oracle", "liboracle.so")
    src = os.path.join(ROOT, "oracle", "ufem_oracle.c")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile")], cwd=ROOT)
    yield
