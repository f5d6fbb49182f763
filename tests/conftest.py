"""Test configuration: the `gpu` marker, fixture paths and the oracle import path."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and liblarmor_b200.so")


@pytest.fixture(scope="session")
def dki_block():
    return dict(np.load(GOLDEN / "dki_block.npz"))


@pytest.fixture(scope="session")
def mfod_fixture():
    return dict(np.load(GOLDEN / "mfod.npz"))


@pytest.fixture(scope="session")
def msmt_fixture():
    return dict(np.load(GOLDEN / "msmt.npz"))


@pytest.fixture(scope="session")
def peaks_fixture():
    return dict(np.load(GOLDEN / "peaks.npz"))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o

    o.lib()
    return o


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch
