import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "_ref", "liboracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True, capture_output=True)


@pytest.fixture(scope="session")
def oracle_lib():
    _ensure_oracle()
    from oracle import orc
    return orc.lib()


@pytest.fixture(scope="session")
def ref_available():
    """The reference build (oracle/_ref/libref_*.so) exists (built where the reference sources are)."""
    d = os.path.join(ROOT, "oracle", "_ref")
    return all(os.path.exists(os.path.join(d, f)) for f in ("libmxshim.so", "libref_mc.so", "libref_heat.so"))
