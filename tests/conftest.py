"""Shared fixtures. GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _make(path: Path, *targets: str) -> None:
    subprocess.run(["make", "-s", "-C", str(path), *targets], check=True,
                   stdout=subprocess.DEVNULL)


@pytest.fixture(scope="session")
def golden():
    def load(name: str):
        return np.load(GOLDEN / name, allow_pickle=False)
    return load


@pytest.fixture(scope="session")
def oracle():
    """The C restatement (oracle/rcpg_oracle.c), built on demand."""
    _make(REPO / "oracle", "oracle")
    from tests import oracle_lib
    return oracle_lib.load()


@pytest.fixture(scope="session")
def hostemu():
    """CPU emulation of the engine's exact mode (tests/hostemu)."""
    _make(REPO / "tests" / "hostemu")
    from tests import hostemu_lib
    return hostemu_lib.load()


@pytest.fixture(scope="session")
def native():
    from rcpgenerator_b200 import _native
    return _native


@pytest.fixture(scope="session")
def cuda_device(native):
    n = native.lib.rcpg_device_count()
    assert n > 0, "GPU test run without a visible CUDA device"
    import torch
    assert torch.cuda.is_available()
    return torch.device("cuda:0")
