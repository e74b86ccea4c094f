"""Shared fixtures.  `gpu` marks tests that need a B200; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _gpu_present() -> bool:
    try:
        import ctypes

        cudart = ctypes.CDLL("libcudart.so")
    except OSError:
        try:
            import torch

            return bool(torch.cuda.is_available())
        except Exception:
            return False
    count = ctypes.c_int(0)
    return cudart.cudaGetDeviceCount(ctypes.byref(count)) == 0 and count.value > 0


GPU_PRESENT = _gpu_present()


@pytest.fixture(scope="session")
def gpu():
    if not GPU_PRESENT:
        pytest.skip("no CUDA device")
    return 0


@pytest.fixture(scope="session")
def ref():
    from oracle.ref import ReferenceLibrary

    try:
        return ReferenceLibrary("cpu")
    except FileNotFoundError as error:
        pytest.skip(str(error))


@pytest.fixture(scope="session")
def golden_dir() -> Path:
    return REPO / "tests" / "golden"
