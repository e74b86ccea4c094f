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


def two_pin_design(first=(1.3, 1.7), second=(6.4, 4.6)):
    """The reference's RUDY fixture (RudyTests.cpp:12-38): two 1x1 modules joined by
    one unit-weight net on a 10 x 10 core (ten unit-height rows of ten unit sites)."""
    import numpy as np

    from myplacement_b200.design import Design

    rows = 10
    return Design(
        module_width=np.ones(2), module_height=np.ones(2), module_x=np.array([first[0], second[0]]),
        module_y=np.array([first[1], second[1]]), module_flags=np.zeros(2), net_weight=np.ones(1),
        net_pin_start=np.array([0, 2]), pin_module=np.array([0, 1]), pin_offset_x=np.zeros(2),
        pin_offset_y=np.zeros(2), row_bottom=np.arange(rows, dtype=float), row_height=np.ones(rows),
        row_site_width=np.ones(rows), row_site_spacing=np.ones(rows), row_x_start=np.zeros(rows),
        row_site_count=np.full(rows, 10), name="rudy_two_pin")
