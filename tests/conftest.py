import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


def _ensure_oracle():
    need = [os.path.join(ROOT, "oracle", n) for n in ("liboracle.so", "liboracle_libm.so")]
    if not all(os.path.exists(p) for p in need):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)


def _ensure_lib():
    from pelemp_b200 import build
    build.build_lib()


_ensure_oracle()
_ensure_lib()


@pytest.fixture(scope="session")
def oracle():
    from oracle.pyoracle import Oracle
    return Oracle(libm=False)


@pytest.fixture(scope="session")
def oracle_libm():
    from oracle.pyoracle import Oracle
    return Oracle(libm=True)
