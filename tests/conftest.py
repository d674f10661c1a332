"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU.

The CPU checkers (the oracle) are built from ``oracle/`` on demand; the
compiled reference (``oracle/_ref``) is only available where it was built
(it needs the reference sources) -- tests that need it skip otherwise.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def port_lib():
    """Builds (if needed) and returns the path of the C restatement."""
    from oracle import ref
    if not os.path.exists(ref.PORT_LIB):
        subprocess.run(["make", "-s", "port"], cwd=os.path.join(ROOT, "oracle"), check=True)
    return ref.PORT_LIB


@pytest.fixture(scope="session")
def ref_available():
    from oracle import ref
    return os.path.exists(ref.REF_LIB)


@pytest.fixture(scope="session")
def engine_lib():
    """The CUDA engine library (built here if the sources are newer)."""
    from sdddst_b200 import build, capi
    build.build()
    capi.load()
    return capi
