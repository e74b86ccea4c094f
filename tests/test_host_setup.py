"""The engine's host setup against the reference's, bit for bit (CPU only).

The session setup -- static density (initializeStaticDensity), fillers
(createDensityFillers, seeded mt19937_64), the preconditioner
(initializePreconditioner) and randomPlacement -- must be identical to the
reference's so that both sides optimize the same problem.
"""
from __future__ import annotations

import numpy as np
import pytest

import myplacement_b200 as mp
from myplacement_b200.design import Design
from oracle.ref import default_options as ref_options


def _fixture(golden_dir, stem):
    f = np.load(golden_dir / "fixtures.npz")
    return Design(**{k[len(stem) + 1:]: f[k] for k in f.files if k.startswith(stem + "_")}, name=stem)


def _cases(golden_dir):
    yield _fixture(golden_dir, "tiny"), 8, 0.85, 100
    yield _fixture(golden_dir, "mixed"), 8, 0.85, 100
    design, bins = mp.workload("small_5k")
    yield design, bins, 0.9, 50_000
    design, bins = mp.workload("mid_210k", scale=0.05)
    yield design, bins, 0.9, 50_000


def test_random_placement_identical(ref, golden_dir):
    for design, *_ in _cases(golden_dir):
        for seed in (0, 2026):
            ax, ay = ref.random_placement(design, seed)
            bx, by = mp.random_placement(design, seed)
            assert np.array_equal(ax, bx) and np.array_equal(ay, by)


def test_session_setup_identical(ref, golden_dir):
    for design, bins, t, fillers in _cases(golden_dir):
        _check_setup(ref, design, bins, t, fillers)


def test_session_setup_identical_at_full_size(ref):
    """The 210k-cell design (848k pins, 260k particles): every set-up loop runs
    on several host threads at this size, and must still match bit for bit."""
    design, bins = mp.workload("mid_210k")
    _check_setup(ref, design, bins, 0.9, 50_000)


def _check_setup(ref, design, bins, t, fillers):
    x, y = mp.random_placement(design, 11)
    design = design.copy_with_positions(x, y)
    rs = ref.session(design, ref_options(bins_x=bins, bins_y=bins, target_density=t, maximum_fillers=fillers))
    mine = mp.host_setup(design, mp.default_options(bins_x=bins, bins_y=bins, target_density=t,
                                                    maximum_fillers=fillers))
    assert mine["particle_count"] == rs.particle_count
    assert mine["movable_count"] == rs.movable_count
    fixed, dark = rs.static_density()
    assert np.array_equal(mine["static_fixed"], fixed)
    assert np.array_equal(mine["static_dark"], dark)
    m = rs.movable_count
    assert np.array_equal(mine["x"][m:], rs.x[m:]) and np.array_equal(mine["y"][m:], rs.y[m:])
    assert np.array_equal(mine["width"], rs.width) and np.array_equal(mine["height"], rs.height)
    assert np.array_equal(mine["layer"], rs.layer)
    # The preconditioner base: pre / raw = base / sqrt(1 + penalty / reference_penalty).
    ev = rs.evaluate(rs.positions, 4.0, 2.0, 1.0, True)
    raw, pre = ev["raw_gradient"][:, 0], ev["preconditioned_gradient"][:, 0]
    ok = np.abs(raw) > 1e-12
    np.testing.assert_allclose(pre[ok] / raw[ok] * np.sqrt(3.0), mine["preconditioner"][ok], rtol=1e-14)


@pytest.mark.parametrize("override,message", [
    (dict(target_density=float("nan")), "non-finite"),
    (dict(feasible_refinement_iterations=0), "outside their valid range"),
    (dict(bins_x=1025, bins_y=1024), "one-million-bin"),
    (dict(iterations=0), "outside their valid range"),
    (dict(backtracking_ratio=1.0), "outside their valid range"),
    (dict(optimizer=0), "adaptive optimizer only"),
    (dict(density_field_boundary=0), "Neumann"),
])
def test_invalid_options_rejected(golden_dir, override, message):
    """validatePublicGlobalOptions / validateAdaptiveOptions (GlobalPlacer.cpp:63-98, AdaptiveGlobalPlacer.cpp:413-454)."""
    design = _fixture(golden_dir, "tiny")
    with pytest.raises(mp.EngineError, match=message) as error:
        mp.host_setup(design, mp.default_options(**{"bins_x": 8, "bins_y": 8, **override}))
    assert error.value.status == mp._abi.MPGP_ERR_INVALID_ARGUMENT


def test_overlapping_rows_rejected(golden_dir):
    """Metrics.cpp:62-70: overlapping SiteRows cannot define the placeable mask."""
    design = _fixture(golden_dir, "tiny")
    fields = {k: getattr(design, k) for k in design.__dataclass_fields__ if not k.startswith("_")}
    for key in ("row_bottom", "row_height", "row_site_width", "row_site_spacing", "row_x_start", "row_site_count"):
        fields[key] = np.concatenate([fields[key], fields[key][:1]])
    with pytest.raises(mp.EngineError, match="Overlapping SiteRows"):
        mp.host_setup(Design(**fields), mp.default_options(bins_x=8, bins_y=8))


def test_malformed_design_rejected(golden_dir):
    design = _fixture(golden_dir, "tiny")
    fields = {k: getattr(design, k) for k in design.__dataclass_fields__ if not k.startswith("_")}
    fields["pin_module"] = fields["pin_module"].copy()
    fields["pin_module"][0] = 99
    with pytest.raises(mp.EngineError, match="unknown module"):
        mp.host_setup(Design(**fields), mp.default_options(bins_x=8, bins_y=8))


def test_defaults_match_reference():
    """mpgp_options_default equals GlobalPlacementOptions' defaults (GlobalPlacer.hpp:26-80)."""
    mine = mp.default_options()
    theirs = ref_options()
    for name, _ in mine._fields_:
        if name in ("compute_backend", "cuda_device", "pad0"):
            continue  # the engine defaults to CUDA on device 0
        assert getattr(mine, name) == getattr(theirs, name), name
