"""The drop-in boundary: the reference's own controller driving the B200 engine.

oracle/_ref/libref_dropin.so is the reference's AdaptiveGlobalPlacer and
GlobalPlacer compiled from their unmodified sources and linked against
myplacement_b200/adapter/mpgp_placement_backend.cpp + libmpgp.so in place of
the reference CUDA backend, so --compute-backend cuda reaches the engine through
tryCreateCudaPlacementBackend / CudaPlacementBackend::evaluate.
"""
from __future__ import annotations


import numpy as np
import pytest

import myplacement_b200 as mp
from myplacement_b200 import _abi
from oracle.ref import ReferenceLibrary, default_options as ref_options

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dropin():
    try:
        return ReferenceLibrary("dropin")
    except FileNotFoundError as error:
        pytest.fail(f"the drop-in build is missing: {error}")


def _case(seed: int = 2026):
    design, bins = mp.workload("small_5k")
    x, y = mp.random_placement(design, seed)
    return design.copy_with_positions(x, y), bins


def test_reference_controller_runs_on_the_engine(gpu, ref, dropin):
    """Same decisions, HPWL and overflow as the reference CPU path for the first 25 iterations."""
    design, bins = _case()
    common = dict(bins_x=bins, bins_y=bins, target_density=0.9, iterations=40,
                  feasible_refinement_iterations=100000, cuda_device=0)
    _, _, cpu_result, cpu_history = ref.global_place(design, ref_options(compute_backend=0, **common))
    x, y, result, history = dropin.global_place(design, ref_options(compute_backend=1, **common))
    assert result.compute_backend_used == _abi.BACKEND_CUDA
    assert result.cuda_device_used == 0
    assert result.completed_iterations == cpu_result.completed_iterations == 40
    for mine, theirs in zip(history[:25], cpu_history[:25]):
        for key in ("accepted", "backtracks", "momentum_restarted"):
            assert mine[key] == theirs[key], (mine["iteration"], key)
        assert mine["hpwl"] == pytest.approx(theirs["hpwl"], rel=1e-4)
        assert mine["overflow"] == pytest.approx(theirs["overflow"], rel=1e-4)
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(y))


def test_reference_auto_backend_selects_the_engine(gpu, dropin):
    """compute_backend=auto picks CUDA when the drop-in reports itself compiled."""
    design, bins = _case(7)
    _, _, result, _ = dropin.global_place(design, ref_options(bins_x=bins, bins_y=bins, target_density=0.9,
                                                              iterations=3, compute_backend=2, cuda_device=0))
    assert result.compute_backend_used == _abi.BACKEND_CUDA
