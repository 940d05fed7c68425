"""Shared test setup: repo on sys.path, the ``gpu`` marker, and the built
libraries (the CPU oracle is rebuilt here if missing; the reference
cross-check build only where the reference tree is present)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# the reference source tree, where this machine has one (LHI_REFERENCE_TREE overrides)
REFERENCE_TREE = os.environ.get("LHI_REFERENCE_TREE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path through the C-ABI)")
    os.environ.setdefault("OMP_NUM_THREADS", "1")  # the reference's OpenMP loops race otherwise


def _make(path, target="all"):
    subprocess.run(["make", "-s", "-C", path, target], check=True, stdout=subprocess.DEVNULL)


@pytest.fixture(scope="session")
def oracle_mod():
    so = os.path.join(ROOT, "oracle", "liblhi_oracle.so")
    if not os.path.exists(so):
        _make(os.path.join(ROOT, "oracle"))
    from oracle import pyoracle
    return pyoracle


@pytest.fixture(scope="session")
def reference_mod(oracle_mod):
    if not oracle_mod.reference_available() and os.path.isdir(REFERENCE_TREE):
        _make(os.path.join(ROOT, "oracle", "refbuild"))
    if not oracle_mod.reference_available():
        pytest.skip("reference cross-check build (oracle/_ref/libref.so) not available")
    return oracle_mod


@pytest.fixture(scope="session")
def lhi():
    so = os.path.join(ROOT, "liquidhairinteration_b200", "liblhi.so")
    if not os.path.exists(so):
        _make(os.path.join(ROOT, "liquidhairinteration_b200"))
    from liquidhairinteration_b200 import _lib
    return _lib
