"""Parity of the B200 engine with the oracle, through the C ABI (needs a GPU).

Tolerances (stated per check):
  * density layers: bit-exact against the fixed-point oracle (oracle/density_fixed.c);
  * per-evaluation gradients: max |g - g_ref| <= 1e-4 * max |g_ref| per component
    set, against the reference CPU path (FP64) at identical positions;
  * scalars (HPWL, smooth wirelength, energy, overflow): 1e-5 relative;
  * DCT field: max |E - E_ref| <= 1e-5 * max |E_ref| against the reference's
    FFTW-definition solver (FP64);
  * whole runs (280-iteration budget, early stop on, 12 seeds x 17 starts): every
    final overflow <= 0.10 and <= the worst reference run's + 0.005; the mean final
    HPWL relative to the reference run of the seed equal to the reference's own
    nudged runs' mean within three standard errors; the first 25 iterations take
    the reference's decisions (see the whole-run tests for why per-run HPWL
    agreement is not a meaningful bound).
"""
from __future__ import annotations

import numpy as np
import pytest

import myplacement_b200 as mp
from myplacement_b200.design import Design
from oracle.ref import ReferenceLibrary, default_options as ref_options, fixed_deposit

pytestmark = pytest.mark.gpu

GRADIENT_TOL = 1e-4
SCALAR_TOL = 1e-5
FIELD_TOL = 1e-5


def _golden(golden_dir):
    g = np.load(golden_dir / "eval_small.npz")
    design = Design(**{k[4:]: g[k] for k in g.files if k.startswith("dsg_")}, name="eval_small")
    return g, design


def _backend_from_golden(g, design):
    bins = int(g["bins"])
    layout = mp.build_layout(design, g["particle_width"], g["particle_height"], g["particle_layer"],
                             g["particle_pin_count"], int(g["movable_count"]), bins, bins, float(g["target_density"]),
                             g["static_fixed"], g["static_dark"])
    backend, reason = mp.try_create_backend(layout, 0)
    assert backend is not None, reason
    return backend, layout


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def test_backend_evaluation_matches_golden(gpu, golden_dir):
    """One CudaPlacementBackend::evaluate against the committed reference outputs."""
    g, design = _golden(golden_dir)
    backend, _ = _backend_from_golden(g, design)
    ev = backend.evaluate(g["positions"], float(g["smoothing"]), True)
    assert ev["hpwl"] == pytest.approx(float(g["hpwl"]), rel=SCALAR_TOL)
    assert ev["smooth_wirelength"] == pytest.approx(float(g["smooth_wirelength"]), rel=SCALAR_TOL)
    assert ev["electrostatic_energy"] == pytest.approx(float(g["density_energy"]), rel=SCALAR_TOL)
    for key, golden in (("optimizer_density", g["optimizer_density"]), ("design_density", g["design_density"])):
        mine = np.array([ev[key][k] for k in mp._abi.DENSITY_METRIC_FIELDS])
        np.testing.assert_allclose(mine, golden, rtol=SCALAR_TOL, atol=1e-9)
    assert _rel(ev["wire_gradient"], g["wire_gradient"]) <= GRADIENT_TOL
    assert _rel(ev["density_gradient"], g["density_gradient"]) <= GRADIENT_TOL


def test_density_layers_bit_exact(gpu, golden_dir):
    """The device scatter equals the fixed-point oracle bit for bit, run after run."""
    g, design = _golden(golden_dir)
    backend, layout = _backend_from_golden(g, design)
    bins = int(g["bins"])
    rng = np.random.default_rng(1)
    for trial in range(3):
        pos = g["positions"] + (rng.normal(0.0, 30.0, g["positions"].shape) if trial else 0.0)
        backend.evaluate(pos, 5.0, False)
        layers = backend.density_layers(bins, bins)
        expected = fixed_deposit(pos[:, 0], pos[:, 1], g["particle_width"], g["particle_height"], g["particle_layer"],
                                 design.core, bins, bins)
        for mine, theirs in zip(layers, expected):
            assert np.array_equal(mine, theirs)
        again = backend.density_layers(bins, bins)
        for a, b in zip(layers, again):
            assert np.array_equal(a, b)


def test_field_matches_reference_solver(gpu, golden_dir, ref):
    """The contraction DCT against the reference ElectrostaticField (FP64) on random and analytic sources."""
    g, design = _golden(golden_dir)
    backend, _ = _backend_from_golden(g, design)
    bins = int(g["bins"])
    region = design.core
    rng = np.random.default_rng(2)
    width, height = region[2] - region[0], region[3] - region[1]
    xc = (np.arange(bins) + 0.5) * width / bins
    yc = (np.arange(bins) + 0.5) * height / bins
    mode = np.cos(np.pi * 2 / width * xc)[None, :] * np.cos(np.pi * 3 / height * yc)[:, None]
    for source in (rng.standard_normal((bins, bins)) + 3.0, mode):
        mine = backend.field_solve(source)
        theirs = ref.field_solve(bins, bins, region, source)
        for a, b in zip(mine, theirs):
            assert _rel(a, b) <= FIELD_TOL


def _session_case(ref, name: str, scale: float, seed: int = 2026):
    design, bins = mp.workload(name, scale=scale)
    x, y = ref.random_placement(design, seed)
    design = design.copy_with_positions(x, y)
    return design, bins


@pytest.mark.parametrize("name,scale", [("small_5k", 1.0), ("mid_210k", 0.1)])
def test_evaluation_parity_against_reference_session(gpu, ref, name, scale):
    """Per-evaluation gradients within 1e-4 of the reference CPU session at identical positions."""
    design, bins = _session_case(ref, name, scale)
    options = ref_options(bins_x=bins, bins_y=bins, target_density=0.9)
    session = ref.session(design, options)
    layout = mp.build_layout(design, session.width, session.height, session.layer, session.pin_count,
                             session.movable_count, bins, bins, 0.9, *session.static_density())
    backend, reason = mp.try_create_backend(layout, 0)
    assert backend is not None, reason
    rng = np.random.default_rng(3)
    pos = session.positions + rng.normal(0.0, 2.0, session.positions.shape)
    width, height = design.core[2] - design.core[0], design.core[3] - design.core[1]
    half = np.stack([session.width, session.height], 1) * 0.5
    pos = np.clip(pos, np.array(design.core[:2]) + half, np.array(design.core[2:]) - half)
    smoothing = 0.75 * max(width, height) / bins
    comp = session.components(pos, smoothing)
    ev = backend.evaluate(pos, smoothing, True)
    assert ev["hpwl"] == pytest.approx(comp["hpwl"], rel=SCALAR_TOL)
    assert ev["smooth_wirelength"] == pytest.approx(comp["smooth_wirelength"], rel=SCALAR_TOL)
    assert ev["electrostatic_energy"] == pytest.approx(comp["energy"], rel=SCALAR_TOL)
    assert _rel(ev["wire_gradient"], comp["wire_gradient"]) <= GRADIENT_TOL
    assert _rel(ev["density_gradient"], comp["density_gradient"]) <= GRADIENT_TOL


def test_wide_grid_evaluation_matches_reference(gpu, ref):
    """A grid wider than the fused metrics-and-split pass takes (4096 x 8 bins): the
    separate metrics and source-split kernels, against the reference session."""
    design, _ = _session_case(ref, "small_5k", 1.0)
    bins_x, bins_y = 4096, 8
    session = ref.session(design, ref_options(bins_x=bins_x, bins_y=bins_y, target_density=0.9))
    layout = mp.build_layout(design, session.width, session.height, session.layer, session.pin_count,
                             session.movable_count, bins_x, bins_y, 0.9, *session.static_density())
    backend, reason = mp.try_create_backend(layout, 0)
    assert backend is not None, reason
    smoothing = 0.75 * max((design.core[2] - design.core[0]) / bins_x, (design.core[3] - design.core[1]) / bins_y)
    comp = session.components(session.positions, smoothing)
    ev = backend.evaluate(session.positions, smoothing, True)
    assert ev["electrostatic_energy"] == pytest.approx(comp["energy"], rel=SCALAR_TOL)
    assert _rel(ev["density_gradient"], comp["density_gradient"]) <= GRADIENT_TOL
    assert _rel(ev["wire_gradient"], comp["wire_gradient"]) <= GRADIENT_TOL


def _nudged(design: Design, bins: int, k: int) -> Design:
    """The same placement with every movable centre moved by at most 1e-6 bin widths
    (the recipe of tests/golden/make_whole_runs.py)."""
    rng = np.random.default_rng(1000 + k)
    step = 1e-6 * (design.core[2] - design.core[0]) / bins
    x = design.module_x.copy()
    y = design.module_y.copy()
    movable = design.movable_mask
    x[movable] += step * rng.uniform(-1.0, 1.0, int(movable.sum()))
    y[movable] += step * rng.uniform(-1.0, 1.0, int(movable.sum()))
    return design.copy_with_positions(x, y)


def _fingerprint(design: Design) -> str:
    parts = [design.module_width, design.module_height, design.module_x, design.module_y, design.pin_offset_x,
             design.pin_offset_y, design.pin_module.astype(np.float64), design.net_pin_start.astype(np.float64)]
    return ",".join(f"{float(np.sum(p * (1.0 + np.arange(p.size) % 7))):.10e}" for p in parts)


def test_early_decisions_match_reference_run(gpu, ref):
    """Decision parity before the trajectories separate: on three seeds the first 25
    iterations take the reference's accept / backtrack / restart decisions with HPWL
    and overflow within 1e-4 (30-iteration runs, early stop off)."""
    for seed in (2026, 7, 11):
        design, bins = _session_case(ref, "small_5k", 1.0, seed=seed)
        fixed = dict(bins_x=bins, bins_y=bins, target_density=0.9, iterations=30,
                     feasible_refinement_iterations=100000)
        _, _, ref_result, ref_history = ref.global_place(design, ref_options(**fixed))
        result = mp.GlobalPlacer().run(design, mp.default_options(**fixed))
        assert result.completed_iterations == ref_result.completed_iterations == 30
        assert result.hpwl_before == pytest.approx(ref_result.hpwl_before, rel=1e-6)
        assert result.overflow_before == pytest.approx(ref_result.overflow_before, rel=1e-6)
        for mine, theirs in zip(result.history[:25], ref_history[:25]):
            for key in ("accepted", "backtracks", "momentum_restarted"):
                assert mine[key] == theirs[key], (seed, mine["iteration"], key)
            assert mine["hpwl"] == pytest.approx(theirs["hpwl"], rel=1e-4)
            assert mine["overflow"] == pytest.approx(theirs["overflow"], rel=1e-4)


def test_whole_runs_match_reference_ensemble(gpu, ref, golden_dir):
    """Whole runs with the reference's default options (280-iteration budget, early stop
    on) on the small design, against the reference CPU runs in tests/golden/whole_runs.json.

    The adaptive controller is chaotic: moving every cell by 1e-6 bin widths changes the
    reference's own final HPWL by about 5 % (standard deviation over the recorded nudged
    runs), in either direction, because the run stops at a different iteration and keeps
    another checkpoint.  A per-run HPWL bound of 0.5 % therefore does not hold even between
    the reference and itself.  What is checked instead, over 12 seeds, each from its
    reference placement and the same 16 nudged placements the reference ran from:
    * every run ends with overflow <= 0.10 and at most 0.005 above the worst reference run
      of its seed;
    * HPWL gaps are taken against the un-nudged reference run of the seed.  The mean gap of
      the engine's runs equals the mean gap of the reference's nudged runs within three
      standard errors of the seed-paired difference, and within 2 % outright;
    * the spread of the engine's gaps is within a factor of two of the reference's.
    """
    import json

    data = json.loads((golden_dir / "whole_runs.json").read_text())
    nudges = min(len(v["nudged"]) for v in data["seeds"].values())
    paired, mine_all, theirs_all = [], [], []
    for seed_text, record in data["seeds"].items():
        seed = int(seed_text)
        design, bins = mp.workload("small_5k")
        x, y = ref.random_placement(design, seed)
        design = design.copy_with_positions(x, y)
        assert _fingerprint(design) == record["fingerprint"], "the synthetic design generator changed"
        base = record["reference"]
        options = mp.default_options(bins_x=bins, bins_y=bins, target_density=0.9)
        worst = max([base["overflow_after"]] + [n["overflow_after"] for n in record["nudged"]])
        gaps = []
        for k in range(-1, nudges):
            start = design if k < 0 else _nudged(design, bins, k)
            result = mp.GlobalPlacer().run(start, options)
            assert result.restored_best_checkpoint == 1
            assert result.overflow_after <= 0.10, (seed, k, result.overflow_after)
            assert result.overflow_after <= worst + 5e-3, (seed, k, result.overflow_after, worst)
            gaps.append(result.hpwl_after / base["hpwl_after"] - 1.0)
        theirs = [n["hpwl_after"] / base["hpwl_after"] - 1.0 for n in record["nudged"][:nudges]]
        paired.append(float(np.mean(gaps)) - float(np.mean(theirs)))
        mine_all.extend(gaps)
        theirs_all.extend(theirs)
    difference = float(np.mean(paired))
    standard_error = float(np.std(paired, ddof=1)) / np.sqrt(len(paired))
    summary = (f"engine mean gap {np.mean(mine_all):+.4%} (std {np.std(mine_all):.3%}), reference nudged "
               f"{np.mean(theirs_all):+.4%} (std {np.std(theirs_all):.3%}), paired difference "
               f"{difference:+.4%} +- {standard_error:.4%}")
    print(summary)
    assert abs(difference) <= 3.0 * standard_error, summary
    assert abs(difference) <= 0.02, summary
    assert 0.5 <= np.std(mine_all) / np.std(theirs_all) <= 2.0, summary


def test_early_stop_run_is_well_formed(gpu, ref):
    """The default run on the small design: early stop, checkpoint restored, cells in the
    core, finite history, initial HPWL and overflow equal to the reference's."""
    design, bins = _session_case(ref, "small_5k", 1.0)
    _, _, ref_long, _ = ref.global_place(
        design, ref_options(bins_x=bins, bins_y=bins, target_density=0.9, iterations=2))
    result = mp.GlobalPlacer().run(design, mp.default_options(bins_x=bins, bins_y=bins, target_density=0.9))
    assert 20 < result.completed_iterations < 280
    assert len(result.history) == result.completed_iterations
    assert result.restored_best_checkpoint == 1
    assert result.overflow_after <= 0.10
    assert result.hpwl_before == pytest.approx(ref_long.hpwl_before, rel=1e-6)
    assert result.overflow_before == pytest.approx(ref_long.overflow_before, rel=1e-6)
    movable = design.movable_mask
    core = design.core
    half_w, half_h = design.module_width[movable] * 0.5, design.module_height[movable] * 0.5
    assert np.all(result.module_x[movable] - half_w >= core[0] - 1e-9)
    assert np.all(result.module_x[movable] + half_w <= core[2] + 1e-9)
    assert np.all(result.module_y[movable] - half_h >= core[1] - 1e-9)
    assert np.all(result.module_y[movable] + half_h <= core[3] + 1e-9)
    for row in result.history:
        assert all(np.isfinite(v) for v in row.values())


def test_global_place_is_deterministic(gpu):
    """Two runs give bit-identical placements (integer scatter, fixed-order reductions)."""
    design, bins = mp.workload("small_5k")
    x, y = mp.random_placement(design, 5)
    design = design.copy_with_positions(x, y)
    options = mp.default_options(bins_x=bins, bins_y=bins, target_density=0.9, iterations=40)
    a = mp.GlobalPlacer().run(design, options)
    b = mp.GlobalPlacer().run(design, options)
    assert np.array_equal(a.module_x, b.module_x) and np.array_equal(a.module_y, b.module_y)
    assert a.history == b.history


@pytest.mark.parametrize("stem", ["tiny", "mixed"])
def test_aggressive_controller_exercises_backtracking_and_restart(gpu, golden_dir, stem):
    """PlacementFlowTests.cpp:198-216: on the reference's fixtures an aggressive controller must
    backtrack and restart momentum (the reference makes 5/5 and 3/3 with these inputs)."""
    f = np.load(golden_dir / "fixtures.npz")
    design = Design(**{k[len(stem) + 1:]: f[k] for k in f.files if k.startswith(stem + "_")}, name=stem)
    x, y = mp.random_placement(design, 2026)
    design = design.copy_with_positions(x, y)
    options = dict(bins_x=8, bins_y=8, iterations=24, maximum_fillers=100, initial_movement_in_bins=1.0,
                   maximum_movement_in_bins=1.0, armijo_coefficient=0.5, objective_increase_for_density=0.0)
    result = mp.GlobalPlacer().run(design, mp.default_options(**options))
    assert result.rejected_candidates > 0
    assert result.momentum_restarts > 0
    assert len(result.history) == result.completed_iterations


def test_fixture_designs_run(gpu, golden_dir):
    """The reference's tiny and mixed fixtures (PlacementFlowTests.cpp:153-164, 311-318) at 8x8 bins."""
    f = np.load(golden_dir / "fixtures.npz")
    for stem, iterations in (("tiny", 24), ("mixed", 16)):
        design = Design(**{k[len(stem) + 1:]: f[k] for k in f.files if k.startswith(stem + "_")}, name=stem)
        x, y = mp.random_placement(design, 2026)
        design = design.copy_with_positions(x, y)
        result = mp.GlobalPlacer().run(design, mp.default_options(bins_x=8, bins_y=8, iterations=iterations,
                                                                  maximum_fillers=100))
        assert result.completed_iterations > 0 and result.accepted_iterations > 0
        assert result.restored_best_checkpoint == 1
        assert len(result.history) == result.completed_iterations


def test_no_movable_modules_returns_empty_result(gpu):
    """AdaptiveGlobalPlacer.cpp:653: a design with nothing movable returns an empty result."""
    design, bins = mp.workload("small_5k")
    flags = design.module_flags.copy()
    flags[:] |= mp._abi.MODULE_FIXED
    fixed = Design(**{**{k: getattr(design, k) for k in design.__dataclass_fields__ if not k.startswith("_")},
                      "module_flags": flags})
    result = mp.GlobalPlacer().run(fixed, mp.default_options(bins_x=bins, bins_y=bins))
    assert result.completed_iterations == 0
    assert np.array_equal(result.module_x, design.module_x)


def test_invalid_smoothing_is_rejected(gpu, golden_dir):
    """CudaPlacementBackend.cu:926-928: non-positive smoothing is an invalid argument."""
    g, design = _golden(golden_dir)
    backend, _ = _backend_from_golden(g, design)
    with pytest.raises(mp.EngineError) as error:
        backend.evaluate(g["positions"], 0.0, True)
    assert error.value.status == mp._abi.MPGP_ERR_INVALID_ARGUMENT


def test_budget_is_enforced(gpu, golden_dir):
    """DeviceMemoryBudget (CudaPlacementBackend.cu:60-79): a tiny budget is refused with a reason."""
    g, design = _golden(golden_dir)
    bins = int(g["bins"])
    layout = mp.build_layout(design, g["particle_width"], g["particle_height"], g["particle_layer"],
                             g["particle_pin_count"], int(g["movable_count"]), bins, bins, 0.9, g["static_fixed"],
                             g["static_dark"])
    backend, reason = mp.try_create_backend(layout, 0, maximum_bytes=4096)
    assert backend is None and "budget" in reason
