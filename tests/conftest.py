"""Shared fixtures. Tests marked `gpu` need a CUDA device and the built library; the rest
run on the CPU (the oracle against the reference, host logic, the library's exports)."""
from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ref_lib():
    from oracle import refworld
    if not refworld.ref_available():
        pytest.skip("oracle/_ref/libnphref.so not built (the reference sources are absent)")
    return refworld


@pytest.fixture(scope="session")
def solver():
    if not cuda_available():
        pytest.skip("no CUDA device")
    from nepheline_b200.solver import Solver
    s = Solver(device=0)
    yield s
    s.close()
