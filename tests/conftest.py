"""Shared test set-up: import paths, the `gpu` marker and device checks.

CPU tests (-m "not gpu") cover the oracle against the reference's known
answers and golden fixtures, the host logic and the C ABI surface.  GPU tests
(-m gpu) compare the CUDA library, called through its C ABI, with the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "amsc-nbody_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


@pytest.fixture(scope="session")
def nbb_mod():
    """The nbb package with libnbb.so loaded; skips only where no GPU
    exists (there the library cannot run, and -m gpu is not selected)."""
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    import nbb

    nbb.load()
    return nbb


@pytest.fixture(scope="session")
def oracle():
    import pyoracle

    pyoracle.lib()
    return pyoracle


def golden(name):
    import numpy as np

    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.fail(f"golden fixture {path} missing (generate with tests/golden/make_golden.py)")
    return dict(np.load(path))
