import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the engine and the oracle when their libraries are missing."""
    import subprocess
    if not os.path.exists(os.path.join(ROOT, "dsm_b200", "libdsm.so")):
        subprocess.run([sys.executable, os.path.join(ROOT, "dsm_b200", "build.py")], check=True)
    if not os.path.exists(os.path.join(ROOT, "oracle", "_build", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
