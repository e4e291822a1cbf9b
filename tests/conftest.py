"""Shared fixtures.  GPU tests carry @pytest.mark.gpu and call libgf through
its C ABI; everything else runs on the CPU."""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import pytest

# libgf's void drop-ins exit(99) on error like the reference unless
# GF_NOEXIT is set; tests want the status instead (also for the reference
# linked with libgf, which never loads the Python package).
os.environ.setdefault("GF_NOEXIT", "1")

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls libgf's C ABI")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(GOLDEN / f"{name}.npz"))
    return load


@pytest.fixture(scope="session")
def restatement():
    from oracle.oracle import Restatement
    return Restatement()


@pytest.fixture(scope="session")
def gf():
    """libgf loaded through ctypes; fails loudly if the library is missing."""
    from galaxyfinder_b200 import _lib
    return _lib.lib()


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected without a CUDA device")
    return torch.device("cuda:0")
