"""The oracle pinned against the reference's own test vectors (CPU only).

The reference CPU path (oracle/_ref/libref_cpu.so, built from the reference
sources with the project's FFTW-subset shim) must reproduce the reference's
known-answer tests: DensityFieldTests.cpp (analytic Neumann modes, DC removal,
zero normal field, 2e-12) and DensityModelTests.cpp (the exact 2x2 course-ePlace
example), and PlacementFlowTests.cpp:305-310 (mixed fixture denominator 540).
The fixed-point density restatement (oracle/density_fixed.c) is then checked
against the reference FP64 map.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle.ref import fixed_deposit, fixed_deposit_rects
from myplacement_b200.design import Design

REGION = (-3.0, 2.0, 5.0, 8.0)  # DensityFieldTests.cpp:18
COLUMNS, ROWS = 16, 12


def _mode_source(mx: int, my: int):
    width, height = REGION[2] - REGION[0], REGION[3] - REGION[1]
    wx, wy = math.pi * mx / width, math.pi * my / height
    xc = (np.arange(COLUMNS) + 0.5) * width / COLUMNS
    yc = (np.arange(ROWS) + 0.5) * height / ROWS
    src = np.cos(wx * xc)[None, :] * np.cos(wy * yc)[:, None]
    return src, wx, wy, xc, yc


@pytest.mark.parametrize("mode", [(2, 3), (0, 3), (2, 0)])
def test_field_analytic_neumann_modes(ref, mode):
    """DensityFieldTests.cpp:27-51 and :68-100 (tolerance 2e-12)."""
    src, wx, wy, xc, yc = _mode_source(*mode)
    den = wx * wx + wy * wy
    potential, field_x, field_y = ref.field_solve(COLUMNS, ROWS, REGION, src)
    cx, cy = np.cos(wx * xc)[None, :], np.cos(wy * yc)[:, None]
    np.testing.assert_allclose(potential, cx * cy / den, rtol=0, atol=2e-12)
    np.testing.assert_allclose(field_x, wx * np.sin(wx * xc)[None, :] * cy / den, rtol=0, atol=2e-12)
    np.testing.assert_allclose(field_y, wy * cx * np.sin(wy * yc)[:, None] / den, rtol=0, atol=2e-12)


def test_field_uniform_source_is_zero(ref):
    """DensityFieldTests.cpp:102-111: DC removal zeroes a uniform source."""
    potential, field_x, field_y = ref.field_solve(COLUMNS, ROWS, REGION, np.full((ROWS, COLUMNS), 7.0))
    for grid in (potential, field_x, field_y):
        assert np.abs(grid).max() <= 2e-12


def test_field_zero_normal_component_on_boundary(ref):
    """DensityFieldTests.cpp:53-66: the sampled normal field vanishes on all four edges."""
    src, *_ = _mode_source(2, 3)
    width, height = REGION[2] - REGION[0], REGION[3] - REGION[1]
    ys = REGION[1] + (np.arange(ROWS) + 0.5) * height / ROWS
    xs = REGION[0] + (np.arange(COLUMNS) + 0.5) * width / COLUMNS
    left = np.stack([np.full(ROWS, REGION[0]), ys], 1)
    right = np.stack([np.full(ROWS, REGION[2]), ys], 1)
    bottom = np.stack([xs, np.full(COLUMNS, REGION[1])], 1)
    top = np.stack([xs, np.full(COLUMNS, REGION[3])], 1)
    sx = ref.field_sample(COLUMNS, ROWS, REGION, src, np.concatenate([left, right]))
    sy = ref.field_sample(COLUMNS, ROWS, REGION, src, np.concatenate([bottom, top]))
    assert np.abs(sx[:, 0]).max() <= 2e-12
    assert np.abs(sy[:, 1]).max() <= 2e-12


def test_field_shim_matches_scipy(ref):
    """The FFT shim's REDFT10/REDFT01/RODFT01 agree with scipy's unnormalized DCT/DST types 2/3."""
    scipy_fft = pytest.importorskip("scipy.fft")
    rng = np.random.default_rng(5)
    for columns, rows in ((16, 12), (33, 20), (64, 64)):
        region = (0.0, 0.0, float(columns), rows * 1.5)
        src = rng.standard_normal((rows, columns))
        potential, field_x, field_y = ref.field_solve(columns, rows, region, src)
        c = scipy_fft.dctn(src - src.mean(), type=2)
        k, l = np.arange(columns), np.arange(rows)
        wx, wy = np.pi * k / region[2], np.pi * l / region[3]
        den = wx[None, :] ** 2 + wy[:, None] ** 2
        den[0, 0] = 1.0
        phi = c / (4 * columns * rows) / den
        phi[0, 0] = 0.0
        p2 = scipy_fft.dct(scipy_fft.dct(phi, type=3, axis=0), type=3, axis=1)
        fx = np.zeros_like(phi)
        fx[:, :-1] = (phi * wx[None, :])[:, 1:]
        ex = scipy_fft.dst(scipy_fft.dct(fx, type=3, axis=0), type=3, axis=1)
        fy = np.zeros_like(phi)
        fy[:-1, :] = (phi * wy[:, None])[1:, :]
        ey = scipy_fft.dct(scipy_fft.dst(fy, type=3, axis=0), type=3, axis=1)
        for a, b in ((potential, p2), (field_x, ex), (field_y, ey)):
            assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_density_model_known_answers(ref):
    """DensityModelTests.cpp:10-51: the exact 2x2 course-ePlace example with t = 0.5."""
    bins, with_fillers, without = ref.density_map(
        (0.0, 0.0, 10.0, 10.0), 2, 2, 0.5, placeable=[(0.0, 0.0, 5.0, 10.0)],
        rects=[(0, 0, 2, 5), (0, 5, 2, 10), (2, 0, 5, 5), (2, 5, 5, 10)], layers=[1, 2, 0, 3])
    assert without["dark_area"] == pytest.approx(50.0, abs=1e-12)
    assert without["placeable_area"] == pytest.approx(50.0, abs=1e-12)
    assert without["normalization_area"] == pytest.approx(15.0, abs=1e-12)
    assert with_fillers["normalization_area"] == pytest.approx(15.0, abs=1e-12)
    assert without["total_charge_area"] == pytest.approx(47.5, abs=1e-12)
    assert with_fillers["total_charge_area"] == pytest.approx(55.0, abs=1e-12)
    assert without["total_overflow_area"] == pytest.approx(5.0, abs=1e-12)
    assert without["normalized_overflow"] == pytest.approx(1.0 / 3.0, abs=1e-12)
    assert bins[0, 1, 4] == pytest.approx(25.0, abs=1e-12)  # at(1, 0).dark_area


def test_density_model_rejects_overlapping_rows(ref):
    """DensityModelTests.cpp:40-49."""
    with pytest.raises(RuntimeError, match="Overlapping SiteRows"):
        ref.density_map((0.0, 0.0, 10.0, 10.0), 2, 2, 0.5, placeable=[(0, 0, 10, 10), (0, 0, 10, 10)], rects=[],
                        layers=[])


def test_mixed_fixture_denominator(ref, golden_dir):
    """PlacementFlowTests.cpp:305-310: the macro is target-scaled in the course denominator (540 at 8x8, 0.85)."""
    design = _fixture(golden_dir, "mixed")
    _, density = ref.design_metrics(design, 8, 8, 0.85)
    assert density["normalization_area"] == pytest.approx(540.0, abs=1e-9)


def test_fixed_point_oracle_matches_reference_map(ref):
    """The fixed-point deposit equals the reference FP64 map within FP32 rounding of the overlap."""
    rng = np.random.default_rng(7)
    region = (0.0, 0.0, 600.0, 1200.0)
    columns, rows = 37, 53
    lo = rng.uniform([-20, -20], [600, 1200], size=(400, 2))
    size = rng.uniform(0.1, 90.0, size=(400, 2))
    rects = np.concatenate([lo, lo + size], 1)
    # Degenerate, edge-aligned and out-of-region rectangles (Metrics.cpp:75-76 clip and skip).
    rects = np.concatenate([rects, [[0, 0, 0, 5], [600, 0, 610, 10], [-50, -50, -10, -10], [0, 0, 600, 1200],
                                    [16.2162162, 0, 32.4324324, 22.6415094]]])
    bins, _, _ = ref.density_map(region, columns, rows, 0.9, placeable=[], rects=rects,
                                 layers=np.full(rects.shape[0], 1))
    fixed = fixed_deposit_rects(rects, region, columns, rows)
    bin_area = (600.0 / columns) * (1200.0 / rows)
    np.testing.assert_allclose(fixed * bin_area * 2.0 ** -32, bins[:, :, 1], rtol=0, atol=2e-6 * bin_area)


def test_fixed_point_oracle_matches_golden_layers(golden_dir):
    """The fixed-point deposit of the committed golden case against the reference's FP64 layers."""
    g = np.load(golden_dir / "eval_small.npz")
    design = _golden_design(g)
    region = design.core
    bins = int(g["bins"])
    pos = g["positions"]
    movable, macro, filler = fixed_deposit(pos[:, 0], pos[:, 1], g["particle_width"], g["particle_height"],
                                           g["particle_layer"], region, bins, bins)
    bin_area = (region[2] - region[0]) * (region[3] - region[1]) / (bins * bins)
    scale = bin_area * 2.0 ** -32
    for fixed, reference in ((movable, g["movable_layer"]), (macro, g["macro_layer"]), (filler, g["filler_layer"])):
        np.testing.assert_allclose(fixed * scale, reference, rtol=0, atol=1e-5 * bin_area)
    # Exact integer conservation: each particle deposits its clipped area once.
    assert int(movable.sum() + macro.sum() + filler.sum()) > 0


def _fixture(golden_dir, stem: str) -> Design:
    f = np.load(golden_dir / "fixtures.npz")
    prefix = f"{stem}_"
    return Design(**{k[len(prefix):]: f[k] for k in f.files if k.startswith(prefix)}, name=stem)


def _golden_design(g) -> Design:
    return Design(**{k[len("dsg_"):]: g[k] for k in g.files if k.startswith("dsg_")}, name="eval_small")


# ---- RUDY (RudyTests.cpp) --------------------------------------------------------------------

RUDY_GRID = dict(columns=5, rows=5, minimum_span=0.01)  # RudyTests.cpp:44-48


def _rudy_session(ref, first=(1.3, 1.7), second=(6.4, 4.6)):
    from conftest import two_pin_design
    from oracle.ref import default_options

    return ref.session(two_pin_design(first, second), default_options(bins_x=4, bins_y=4, target_density=0.9))


def _finite_difference(session, positions, particle, axis, capacity, model, delta=1e-5):
    plus, minus = positions.copy(), positions.copy()
    plus[particle, axis] += delta
    minus[particle, axis] -= delta
    e_plus = session.rudy(plus, model=model, capacity=capacity, **RUDY_GRID)["energy"]
    e_minus = session.rudy(minus, model=model, capacity=capacity, **RUDY_GRID)["energy"]
    return (e_plus - e_minus) / (2.0 * delta)


def test_rudy_reference_known_answers(ref):
    """RudyTests.cpp:50-110: demand integrates to the net spans (5.1, 2.9), a 0.45 x mean
    capacity exposes a hotspot, and the analytical gradient of every penalty model agrees
    with a central difference to 3e-6."""
    session = _rudy_session(ref)
    pos = session.positions
    raw = session.rudy(pos, model=1, **RUDY_GRID)
    assert raw["horizontal_total"] == pytest.approx(5.1, abs=1e-12)
    assert raw["vertical_total"] == pytest.approx(2.9, abs=1e-12)
    capacity = (0.45 * raw["horizontal_mean"], 0.45 * raw["vertical_mean"])
    for model in (1, 2, 3):
        ev = session.rudy(pos, model=model, capacity=capacity, gradient=True, **RUDY_GRID)
        assert np.isfinite(ev["energy"]) and ev["energy"] > 0.0
        assert ev["maximum_utilization"] > 1.0
        for axis in (0, 1):
            fd = _finite_difference(session, pos, 0, axis, capacity, model)
            assert ev["gradient"][0, axis] == pytest.approx(fd, abs=3e-6), (model, axis)
    assert abs(session.rudy(pos, model=3, capacity=capacity, gradient=True, **RUDY_GRID)["gradient"][0, 0]) > 1e-10


def test_rudy_reference_boundary_and_degenerate_nets(ref):
    """RudyTests.cpp:112-148: a net whose box edges lie on grid lines keeps a non-zero
    Clarke subgradient; a zero-span net keeps its translation gradient."""
    session = _rudy_session(ref, first=(2.0, 1.7), second=(6.0, 4.6))
    pos = session.positions
    raw = session.rudy(pos, model=2, **RUDY_GRID)
    capacity = (0.45 * raw["horizontal_mean"], 0.45 * raw["vertical_mean"])
    ev = session.rudy(pos, model=2, capacity=capacity, gradient=True, **RUDY_GRID)
    assert abs(ev["gradient"][0, 0]) + abs(ev["gradient"][1, 0]) > 1e-10

    session = _rudy_session(ref)
    pos = session.positions
    raw = session.rudy(pos, model=2, **RUDY_GRID)
    capacity = (0.45 * raw["horizontal_mean"], 0.45 * raw["vertical_mean"])
    pos[1] = pos[0]
    ev = session.rudy(pos, model=2, capacity=capacity, gradient=True, **RUDY_GRID)
    assert np.isfinite(ev["energy"])
    plus, minus = pos.copy(), pos.copy()
    plus[:2, 0] += 1e-5
    minus[:2, 0] -= 1e-5
    fd = (session.rudy(plus, model=2, capacity=capacity, **RUDY_GRID)["energy"] -
          session.rudy(minus, model=2, capacity=capacity, **RUDY_GRID)["energy"]) / 2e-5
    assert ev["gradient"][0, 0] + ev["gradient"][1, 0] == pytest.approx(fd, abs=3e-6)


def test_rudy_reference_rejects_partial_capacity(ref):
    """RudyTests.cpp:150-166: a capacity with one zero component is refused."""
    session = _rudy_session(ref)
    with pytest.raises(RuntimeError):
        session.rudy(session.positions, model=1, capacity=(1.0, 0.0), **RUDY_GRID)
