"""Shared pytest setup: markers, import paths and the CPU oracle builds."""

from __future__ import annotations

import pathlib
import sys

import pytest

REPO = pathlib.Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO / "tide-gpr_b200"))
sys.path.insert(0, str(REPO / "tests"))
GOLDEN = REPO / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libtide_b200.so")
    config.addinivalue_line("markers", "slow: longer CPU or GPU runs")


@pytest.fixture(scope="session")
def oracle():
    from oracle_harness import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
