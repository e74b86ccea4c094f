"""Detailed placement (window reordering on the device) against the reference's CUDA backend.

The reference backend (src/placement/cuda/CudaDetailedPlacementBackend.cu,
compiled for sm_100a into oracle/_ref/libref_cuda.so and run through
DetailedPlacer::run) and this engine see the same legal placements.  The
final centres and orientations must be bit-identical and so must every counter
of DetailedPlacementResult (windows, permutations, accepted operations,
passes) and both HPWL values.  The drop-in (the reference's DetailedPlacer
over myplacement_b200/adapter/mpgp_detailed_placement_backend.cpp,
oracle/_ref/libref_dropin.so) must give the same again.  Where the reference
backend declines, the engine declines with the same reason.
"""
from __future__ import annotations

import numpy as np
import pytest

import myplacement_b200 as mp
from myplacement_b200 import _abi
from myplacement_b200.design import packed_placement
from oracle.ref import ReferenceFailure, ReferenceLibrary

CPU, CUDA = 0, 1


def _bits(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def _fixture() -> mp.Design:
    """Four 5 x 10 cells in the order A, C, D, B on one row, nets AB and CD: only a
    coordinated reorder of all four (to A, B, C, D) improves the HPWL (to 10)."""
    x = np.array([0.0, 5.0, 10.0, 15.0]) + 2.5
    return mp.Design(module_width=np.full(4, 5.0), module_height=np.full(4, 10.0), module_x=x,
                     module_y=np.full(4, 5.0), module_flags=np.zeros(4, np.int32), net_weight=np.ones(2),
                     net_pin_start=np.array([0, 2, 4]), pin_module=np.array([0, 3, 1, 2]),
                     pin_offset_x=np.zeros(4), pin_offset_y=np.zeros(4), row_bottom=np.zeros(1),
                     row_height=np.full(1, 10.0), row_site_width=np.ones(1), row_site_spacing=np.ones(1),
                     row_x_start=np.zeros(1), row_site_count=np.array([40]))


def _legal_case(seed: int, cells: int, spacing: float = 1.0,
                fractional: bool = False) -> tuple[mp.Design, np.ndarray]:
    """A synthetic design (terminals, fixed macros, degree-2..64 nets) packed legally
    into its rows; random module and row orientations, real-valued pin offsets
    and net weights; with `fractional`, real cell widths on a `spacing` site grid."""
    rng = np.random.default_rng(seed)
    design = mp.synthetic_design(cells=cells, nets=int(cells * 1.04), terminals=max(8, cells // 50),
                                 macros=max(1, cells // 2000), seed=seed, name=f"legal{seed}")
    if fractional:
        design.module_width[:cells] = np.round(rng.uniform(0.6, 6.5, cells), 3)
        design.row_site_spacing[:] = spacing
        design.row_site_count[:] = np.ceil(design.row_site_count / spacing).astype(np.int64)
    half_w = design.module_width[design.pin_module] * 0.5
    half_h = design.module_height[design.pin_module] * 0.5
    design.pin_offset_x[:] = rng.uniform(-1.0, 1.0, design.pin_count) * half_w
    design.pin_offset_y[:] = rng.uniform(-1.0, 1.0, design.pin_count) * half_h
    design.net_weight[:] = rng.choice([1.0, 0.5, 2.0, 1.25], design.net_count)
    placed = packed_placement(design, seed + 1, gap_probability=0.08)
    placed.module_orientation = rng.integers(0, 8, design.module_count).astype(np.int32)
    rows = rng.integers(0, 9, design.row_bottom.shape[0]).astype(np.int32)
    return placed, rows


def _assert_legal(before: mp.Design, after_x: np.ndarray, after_y: np.ndarray) -> None:
    """Every cell stays on its row, on the site grid of the window it moved in, without overlaps."""
    assert np.array_equal(_bits(after_y), _bits(before.module_y))
    movable = (before.module_flags & (_abi.MODULE_TERMINAL | _abi.MODULE_FIXED)) == 0
    for y in np.unique(before.module_y[movable]):
        on_row = np.nonzero(movable & (before.module_y == y))[0]
        left = after_x[on_row] - before.module_width[on_row] * 0.5
        order = np.argsort(left, kind="stable")
        right = left[order] + before.module_width[on_row][order]
        assert np.all(right[:-1] <= left[order][1:] + 1e-9)


@pytest.fixture(scope="module")
def libraries():
    return ReferenceLibrary("cuda"), ReferenceLibrary("dropin")


# ---- without a device ------------------------------------------------------------------------


def test_declines_like_reference_without_running(libraries):
    """Options the reference backend does not take are refused with its reason, before any device work."""
    reference, _ = libraries
    design = _fixture()
    for change, reason in (({"window_size": 3}, "four-cell window only"), ({"method": 1}, "four-cell window only"),
                           ({"passes": 0}, "outside their valid range"),
                           ({"maximum_net_degree": 1}, "outside their valid range"),
                           ({"improvement_epsilon": -1.0}, "outside their valid range")):
        options = mp.default_detailed_options(**change)
        with pytest.raises(mp.EngineError) as mine:
            mp.DetailedPlacer().run(design, options)
        assert mine.value.status == _abi.MPGP_ERR_UNAVAILABLE
        assert reason in str(mine.value)
        if "window_size" not in change:
            continue  # DetailedPlacer::run changes the method or rejects these before its backend is asked
        with pytest.raises(ReferenceFailure) as theirs:
            reference.detailed_place(design, options, CUDA)
        assert theirs.value.message.endswith(str(mine.value).split(": ", 1)[1])


def test_defaults_follow_the_reference():
    """DetailedPlacementOptions (DetailedPlacer.hpp:23-44): the reference's defaults,
    with the window reorder selected and device 0."""
    o = mp.default_detailed_options()
    assert (o.method, o.passes, o.window_size, o.maximum_net_degree) == (_abi.DETAILED_WINDOW_REORDER, 2, 4, 64)
    assert o.improvement_epsilon == 1e-9 and o.maximum_cuda_memory_bytes == 2 << 30 and o.cuda_device == 0


def test_invalid_orientations_are_rejected():
    design = _fixture()
    design.module_orientation = np.array([0, 9, 0, 0], np.int32)
    with pytest.raises(mp.EngineError) as error:
        mp.DetailedPlacer().run(design)
    assert error.value.status == _abi.MPGP_ERR_INVALID_ARGUMENT
    with pytest.raises(mp.EngineError) as error:
        mp.DetailedPlacer().run(_fixture(), row_orientation=np.array([-1], np.int32))
    assert error.value.status == _abi.MPGP_ERR_INVALID_ARGUMENT


def test_no_cpu_fallback_without_gpu():
    from conftest import GPU_PRESENT
    if GPU_PRESENT:
        pytest.skip("checks the behaviour without a GPU")
    with pytest.raises(mp.EngineError) as error:
        mp.DetailedPlacer().run(_fixture())
    assert error.value.status == _abi.MPGP_ERR_UNAVAILABLE
    assert "unavailable on this host" in str(error.value)


@pytest.mark.parametrize("spacing,fractional", [(1.0, False), (0.19, True), (0.5, True)])
def test_packed_placement_is_legal(spacing, fractional):
    design, _ = _legal_case(3, 2000, spacing=spacing, fractional=fractional)
    _assert_legal(design, design.module_x, design.module_y)


# ---- on the device ------------------------------------------------------------------------------


@pytest.mark.gpu
def test_fixture_takes_the_coordinated_reorder(gpu, libraries):
    """DetailedPlacementTests.cpp:49-63 on the device backend: one accepted
    operation, 24 orders evaluated, final HPWL 10."""
    reference, dropin = libraries
    options = mp.default_detailed_options(passes=1)
    placed, result = mp.DetailedPlacer().run(_fixture(), options)
    assert result["accepted_operations"] == 1 and result["evaluated_permutations"] == 24
    assert result["hpwl_after"] == 10.0 and result["hpwl_before"] > 10.0
    x, y, orientation, theirs, used = reference.detailed_place(_fixture(), options, CUDA)
    assert used == CUDA
    assert np.array_equal(_bits(placed.module_x), _bits(x)) and np.array_equal(placed.module_orientation, orientation)
    for key in ("hpwl_before", "hpwl_after", "evaluated_windows", "evaluated_permutations", "accepted_operations",
                "completed_passes"):
        assert result[key] == theirs[key], key
    assert dropin.detailed_place(_fixture(), options, CUDA)[4] == CUDA


CASES = [
    dict(seed=11, cells=3000),
    dict(seed=12, cells=6000),
    dict(seed=13, cells=3000, spacing=0.19, fractional=True),
    dict(seed=14, cells=4000, spacing=0.5, fractional=True),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("passes,degree", [(2, 64), (3, 4)])
def test_matches_reference_cuda_backend(gpu, libraries, case, passes, degree):
    """Bit-identical centres, orientations, HPWLs and counters against the
    reference backend, through the C ABI and through the drop-in; a degree limit
    of 4 sends many windows down the host rule as well."""
    reference, dropin = libraries
    design, rows = _legal_case(**CASES[case])
    options = mp.default_detailed_options(passes=passes, maximum_net_degree=degree)
    placed, mine = mp.DetailedPlacer().run(design, options, row_orientation=rows)
    x, y, orientation, theirs, used = reference.detailed_place(design, options, CUDA, rows)
    assert used == CUDA
    assert mine["accepted_operations"] > 0
    for key in ("hpwl_before", "hpwl_after", "evaluated_windows", "evaluated_permutations", "accepted_operations",
                "completed_passes"):
        assert mine[key] == theirs[key], (key, mine[key], theirs[key])
    assert np.array_equal(_bits(placed.module_x), _bits(x))
    assert np.array_equal(_bits(placed.module_y), _bits(y))
    assert np.array_equal(placed.module_orientation, orientation)
    assert mine["hpwl_after"] < mine["hpwl_before"]
    _assert_legal(design, placed.module_x, placed.module_y)
    dx, dy, dorientation, via_dropin, dused = dropin.detailed_place(design, options, CUDA, rows)
    assert dused == CUDA
    assert np.array_equal(_bits(dx), _bits(x)) and np.array_equal(dorientation, orientation)
    assert via_dropin["accepted_operations"] == theirs["accepted_operations"]
