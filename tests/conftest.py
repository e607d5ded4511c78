import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _build_oracle():
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), os.path.join(ROOT, "oracle", "liboracle.so")],
                   check=True)


@pytest.fixture(scope="session", autouse=True)
def oracle_built():
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        _build_oracle()
    yield
