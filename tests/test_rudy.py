"""The RUDY routability term on the device against the reference CPU path (needs a GPU).

The engine's demand maps are fixed-point (units of bin_w * 2^-32 and
bin_h * 2^-32, integer atomics) and its pin offsets are FP32, so against the
reference's FP64 evaluateRudy (Rudy.cpp:227-456) at identical positions:
  * demand totals and means within 1e-8 relative, the capacities exact;
  * energy, proxy overflow, maximum and p95 utilisation within 1e-6 relative;
  * the per-particle subgradient within 1e-6 * max |g_ref| (the controller's
    gradient bound is 1e-4);
and whole runs with the term on take the reference's activation iteration, its
first 25 accept / backtrack / restart decisions, HPWL within 1e-4 and the
routability weight within 1e-4 over those rows.
"""
from __future__ import annotations

import numpy as np
import pytest

import myplacement_b200 as mp
from conftest import two_pin_design
from oracle.ref import default_options as ref_options

pytestmark = pytest.mark.gpu

DEMAND_TOL = 1e-8
METRIC_TOL = 1e-6
GRADIENT_TOL = 1e-6
MODELS = {"hinge_l2": mp._abi.RUDY_HINGE_L2, "softplus_l2": mp._abi.RUDY_SOFTPLUS_L2,
          "hinge_l4": mp._abi.RUDY_HINGE_L4}


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def _pair(ref, design, bins, target_density=0.9):
    session = ref.session(design, ref_options(bins_x=bins, bins_y=bins, target_density=target_density))
    layout = mp.build_layout(design, session.width, session.height, session.layer, session.pin_count,
                             session.movable_count, bins, bins, target_density, *session.static_density())
    backend, reason = mp.try_create_backend(layout, 0)
    assert backend is not None, reason
    return session, backend


def _grid_options(columns, rows, model, minimum_span=0.25):
    o = mp.default_options()
    o.rudy_columns, o.rudy_rows, o.rudy_penalty_model = columns, rows, model
    o.rudy_minimum_span_in_bins = minimum_span
    return o


def _compare(session, backend, pos, columns, rows, model, factor, minimum_span=0.25):
    """One raw (no capacity) and one penalised evaluation on both sides; returns the reference's."""
    grid = dict(columns=columns, rows=rows, minimum_span=minimum_span)
    options = _grid_options(columns, rows, model, minimum_span)
    theirs_raw = session.rudy(pos, model=model, **grid)
    mine_raw = backend.rudy(pos, options)
    for key in ("horizontal_total", "vertical_total", "horizontal_mean", "vertical_mean"):
        assert mine_raw[key] == pytest.approx(theirs_raw[key], rel=DEMAND_TOL), key
    capacity = (factor * theirs_raw["horizontal_mean"], factor * theirs_raw["vertical_mean"])
    theirs = session.rudy(pos, model=model, capacity=capacity, gradient=True, **grid)
    mine = backend.rudy(pos, options, capacity=capacity, gradient=True)
    assert mine["horizontal_capacity"] == theirs["horizontal_capacity"]
    assert mine["vertical_capacity"] == theirs["vertical_capacity"]
    for key in ("energy", "proxy_overflow", "maximum_utilization", "p95_utilization"):
        assert mine[key] == pytest.approx(theirs[key], rel=METRIC_TOL, abs=1e-300), key
    assert mine["evaluation_energy"] == pytest.approx(mine["energy"], rel=1e-12)
    if np.abs(theirs["gradient"]).max() > 0.0:
        assert _rel(mine["gradient"], theirs["gradient"]) <= GRADIENT_TOL
    else:
        assert np.abs(mine["gradient"]).max() == 0.0
    return theirs, mine


@pytest.mark.parametrize("model", list(MODELS))
def test_two_pin_fixture_matches_reference(gpu, ref, model):
    """RudyTests.cpp's fixture: totals 5.1 / 2.9, a hotspot at 0.45 x mean, the gradient of each model."""
    session, backend = _pair(ref, two_pin_design(), 4)
    theirs, mine = _compare(session, backend, session.positions, 5, 5, MODELS[model], 0.45, minimum_span=0.01)
    raw = backend.rudy(session.positions, _grid_options(5, 5, MODELS[model], 0.01))
    assert raw["horizontal_total"] == pytest.approx(5.1, abs=DEMAND_TOL)
    assert raw["vertical_total"] == pytest.approx(2.9, abs=DEMAND_TOL)
    assert mine["maximum_utilization"] > 1.0
    assert np.abs(mine["gradient"][0]).max() > 1e-10


def test_grid_line_and_degenerate_nets_match_reference(gpu, ref):
    """Box edges exactly on grid lines (the Clarke subgradient split) and a zero-span net."""
    session, backend = _pair(ref, two_pin_design((2.0, 1.7), (6.0, 4.6)), 4)
    _, mine = _compare(session, backend, session.positions, 5, 5, MODELS["softplus_l2"], 0.45, minimum_span=0.01)
    assert abs(mine["gradient"][0, 0]) + abs(mine["gradient"][1, 0]) > 1e-10
    session, backend = _pair(ref, two_pin_design(), 4)
    pos = session.positions.copy()
    pos[1] = pos[0]
    _compare(session, backend, pos, 5, 5, MODELS["softplus_l2"], 0.45, minimum_span=0.01)


@pytest.mark.parametrize("name,scale,model", [("small_5k", 1.0, "hinge_l2"), ("small_5k", 1.0, "softplus_l2"),
                                              ("small_5k", 1.0, "hinge_l4"), ("mid_210k", 0.1, "hinge_l2")])
def test_synthetic_designs_match_reference(gpu, ref, name, scale, model):
    """Thousands of nets (fixed-pin nets and macros included) at random positions, 64 x 64 and 48 x 48 grids."""
    design, bins = mp.workload(name, scale=scale)
    x, y = mp.random_placement(design, 2026)
    design = design.copy_with_positions(x, y)
    session, backend = _pair(ref, design, bins)
    rng = np.random.default_rng(4)
    pos = session.positions + rng.normal(0.0, 2.0, session.positions.shape)
    half = np.stack([session.width, session.height], 1) * 0.5
    pos = np.clip(pos, np.array(design.core[:2]) + half, np.array(design.core[2:]) - half)
    theirs, _ = _compare(session, backend, pos, 64, 64, MODELS[model], 0.8)
    assert theirs["proxy_overflow"] > 0.0  # the capacity exposes hotspots
    # A second grid through a fresh backend (the first call fixes a backend's grid).
    session2, backend2 = _pair(ref, design, bins)
    _compare(session2, backend2, pos, 48, 48, MODELS[model], 1.0)


def test_backend_grid_is_fixed_by_first_use(gpu, ref):
    session, backend = _pair(ref, two_pin_design(), 4)
    backend.rudy(session.positions, _grid_options(5, 5, 1, 0.01))
    with pytest.raises(mp.EngineError):
        backend.rudy(session.positions, _grid_options(6, 6, 1, 0.01))


def _rudy_run_options(factory, bins, start):
    return factory(bins_x=bins, bins_y=bins, target_density=0.9, iterations=60,
                   feasible_refinement_iterations=100000, rudy_penalty_model=1, routability_start_overflow=start,
                   rudy_validation_bins=48)


@pytest.mark.parametrize("start", [0.5, 0.1])
def test_run_with_routability_matches_reference(gpu, ref, start):
    """Whole runs with the RUDY term: activation at the initial placement (start 0.5) and
    mid-run (start 0.1, iteration 3 on this design) as the reference CPU run does."""
    design, bins = mp.workload("small_5k")
    x, y = mp.random_placement(design, 2026)
    design = design.copy_with_positions(x, y)
    _, _, ref_result, ref_history = ref.global_place(design, _rudy_run_options(ref_options, bins, start))
    result = mp.GlobalPlacer().run(design, _rudy_run_options(mp.default_options, bins, start))
    first = lambda history: next(row["iteration"] for row in history if row["rudy_active"])
    assert first(result.history) == first(ref_history)
    for mine, theirs in zip(result.history[:25], ref_history[:25]):
        for key in ("accepted", "backtracks", "momentum_restarted", "rudy_active"):
            assert mine[key] == theirs[key], (mine["iteration"], key)
        assert mine["hpwl"] == pytest.approx(theirs["hpwl"], rel=1e-4)
        assert mine["rudy_weight"] == pytest.approx(theirs["rudy_weight"], rel=1e-4)
        assert mine["rudy_energy"] == pytest.approx(theirs["rudy_energy"], rel=1e-3, abs=1e-12)
    assert result.rudy_horizontal_capacity == pytest.approx(ref_result.rudy_horizontal_capacity, rel=1e-4)
    assert result.rudy_vertical_capacity == pytest.approx(ref_result.rudy_vertical_capacity, rel=1e-4)
    for key in ("rudy_energy_after", "rudy_proxy_overflow_after", "rudy_maximum_utilization_after",
                "rudy_p95_utilization_after", "rudy_validation_energy_after",
                "rudy_validation_p95_utilization_after"):
        value = getattr(result, key)
        assert np.isfinite(value) and value >= 0.0, key
    assert result.rudy_p95_utilization_after > 0.0 and result.rudy_validation_p95_utilization_after > 0.0
    assert result.completed_iterations == ref_result.completed_iterations


def test_routability_run_is_deterministic(gpu):
    design, bins = mp.workload("small_5k")
    x, y = mp.random_placement(design, 9)
    design = design.copy_with_positions(x, y)
    options = _rudy_run_options(mp.default_options, bins, 0.5)
    options.iterations = 30
    a = mp.GlobalPlacer().run(design, options)
    b = mp.GlobalPlacer().run(design, options)
    assert np.array_equal(a.module_x, b.module_x) and np.array_equal(a.module_y, b.module_y)
    assert a.history == b.history
    assert a.rudy_energy_after == b.rudy_energy_after
