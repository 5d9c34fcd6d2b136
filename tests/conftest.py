import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")
    # the CPU oracle is test infrastructure: make sure it is built
    if not os.path.exists(os.path.join(ROOT, "oracle", "liborc.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


@pytest.fixture(scope="session")
def small_case():
    from elastic_isotropic_operators_b200 import synthetic
    return synthetic.small()
