"""Shared test set-up.

Markers: ``gpu`` -- needs a CUDA device (run with ``-m gpu`` on a B200).
The CPU oracle (oracle/) is the checker; the product never imports it.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def psx():
    """The product library (built in-tree if missing)."""
    from peasoup_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from peasoup_b200.build import build
        build()
    return _lib.load()


@pytest.fixture(scope="session")
def ref_host():
    """The reference's own host classes, built from its sources (skipped
    where neither the built library nor the sources exist)."""
    from oracle import oracle as O
    if not os.path.exists(O.REF_HOST_PATH):
        try:
            O.build_reference()
        except Exception:
            pass
    if not os.path.exists(O.REF_HOST_PATH):
        pytest.skip("reference host library not built")
    O.ref_host()
    return O


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="session")
def ref_gpu(cuda):
    """The reference's own CUDA build (oracle/_ref); skipped if not built."""
    from oracle import oracle as O
    if not os.path.exists(O.REF_GPU_PATH):
        pytest.skip("reference GPU library not built")
    O.ref_gpu()
    return O
