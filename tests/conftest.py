import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "stomakhin-style-snow-simulator_b200")
for p in (PKG, os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def oracle():
    """The CPU restatement (built from oracle/ if needed)."""
    from oracle_lib import ORACLE_SO, Oracle

    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so", "oracle_tests"],
                       check=True, capture_output=True)
    return Oracle()


@pytest.fixture(scope="session")
def snow():
    """The CUDA library on device 0 (fails, never skips, if it is not built)."""
    import snow_b200

    snow_b200.init(0)
    return snow_b200
