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


def pytest_runtest_logreport(report):
    """With DSM_TEST_TIMES set to a path, each test's call time and outcome
    are appended to that file as the test ends (readable even when the run is
    cut short)."""
    path = os.environ.get("DSM_TEST_TIMES")
    if path and report.when == "call":
        with open(path, "a") as f:
            f.write(f"{report.duration:9.2f} {report.outcome:7s} {report.nodeid}\n")
