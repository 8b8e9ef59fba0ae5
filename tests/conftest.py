"""Shared test fixtures.

Markers: `gpu` tests need a CUDA device and call the library through its C ABI;
everything else runs on CPU. The checker libraries (oracle/_build, oracle/_ref)
are built on demand when their sources are present."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

REF_APP = os.path.join(ROOT, "oracle", "_ref", "idx2App")
REF_HARNESS = os.path.join(ROOT, "oracle", "_ref", "libidx2_ref_harness.so")
ORACLE_LIB = os.path.join(ROOT, "oracle", "_build", "libidx2_oracle.so")
IDX2G_LIB = os.path.join(ROOT, "idx2_b200", "libidx2g.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_lib():
    if not os.path.exists(ORACLE_LIB):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "port"], check=True,
                       capture_output=True)
    import ctypes
    return ctypes.CDLL(ORACLE_LIB)


@pytest.fixture(scope="session")
def ref_harness():
    if not os.path.exists(REF_HARNESS):
        pytest.skip("reference harness not built (oracle/_ref)")
    import ctypes
    return ctypes.CDLL(REF_HARNESS)


@pytest.fixture(scope="session")
def ref_app():
    if not os.path.exists(REF_APP):
        pytest.skip("reference CLI not built (oracle/_ref)")
    return REF_APP


@pytest.fixture(scope="session")
def idx2g():
    if not os.path.exists(IDX2G_LIB):
        subprocess.run(["make", "-C", os.path.join(ROOT, "idx2_b200", "csrc"), "-j8"], check=True,
                       capture_output=True)
    import idx2_b200
    return idx2_b200
