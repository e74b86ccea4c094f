"""The precision configuration at full size: 1.3M cells, 2,000 macros, 1.4M nets
(5.5M pins), 1024 x 1024 bins, RUDY at capacity 1.2 x mean demand (needs a GPU).

Against the reference CPU path (FP64) at identical positions:
  * HPWL, smooth wirelength and density energy within 1e-5 relative;
  * wire and density gradients within 1e-4 * max |g_ref|;
  * the Neumann field within 1e-5 * max |E_ref|;
  * RUDY totals within 1e-8, energy and utilisation statistics within 1e-6,
    the subgradient within 1e-6 * max |g_ref|.
The reference takes about a minute of CPU time here (most of it its RUDY
subgradient, which visits every bin of every net's box).
"""
from __future__ import annotations

import numpy as np
import pytest

import myplacement_b200 as mp
from oracle.ref import default_options as ref_options

pytestmark = pytest.mark.gpu

SCALAR_TOL = 1e-5
GRADIENT_TOL = 1e-4
FIELD_TOL = 1e-5


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.fixture(scope="module")
def large(ref):
    design, bins = mp.workload("large_1m3")
    x, y = mp.random_placement(design, 2026)
    design = design.copy_with_positions(x, y)
    session = ref.session(design, ref_options(bins_x=bins, bins_y=bins, target_density=0.9))
    layout = mp.build_layout(design, session.width, session.height, session.layer, session.pin_count,
                             session.movable_count, bins, bins, 0.9, *session.static_density())
    backend, reason = mp.try_create_backend(layout, 0)
    assert backend is not None, reason
    rng = np.random.default_rng(5)
    pos = session.positions + rng.normal(0.0, 4.0, session.positions.shape)
    half = np.stack([session.width, session.height], 1) * 0.5
    pos = np.clip(pos, np.array(design.core[:2]) + half, np.array(design.core[2:]) - half)
    return design, bins, session, backend, pos


def test_large_evaluation_matches_reference(gpu, large):
    design, bins, session, backend, pos = large
    assert session.particle_count == 1_350_000 and bins == 1024
    smoothing = 0.75 * max(design.core[2] - design.core[0], design.core[3] - design.core[1]) / bins
    comp = session.components(pos, smoothing)
    ev = backend.evaluate(pos, smoothing, True)
    assert ev["hpwl"] == pytest.approx(comp["hpwl"], rel=SCALAR_TOL)
    assert ev["smooth_wirelength"] == pytest.approx(comp["smooth_wirelength"], rel=SCALAR_TOL)
    assert ev["electrostatic_energy"] == pytest.approx(comp["energy"], rel=SCALAR_TOL)
    assert _rel(ev["wire_gradient"], comp["wire_gradient"]) <= GRADIENT_TOL
    assert _rel(ev["density_gradient"], comp["density_gradient"]) <= GRADIENT_TOL


def test_large_field_matches_reference(gpu, ref, large):
    design, bins, _, backend, _ = large
    rng = np.random.default_rng(6)
    source = np.abs(rng.standard_normal((bins, bins))) ** 3  # heavy-tailed, like a density map
    mine = backend.field_solve(source)
    theirs = ref.field_solve(bins, bins, design.core, source)
    for a, b in zip(mine, theirs):
        assert _rel(a, b) <= FIELD_TOL


def test_large_routability_matches_reference(gpu, large):
    _, _, session, backend, pos = large
    options = mp.default_options()
    options.rudy_penalty_model = mp._abi.RUDY_HINGE_L2
    raw_ref = session.rudy(pos, 64, 64, options.rudy_penalty_model)
    raw = backend.rudy(pos, options)
    for key in ("horizontal_total", "vertical_total", "horizontal_mean", "vertical_mean"):
        assert raw[key] == pytest.approx(raw_ref[key], rel=1e-8), key
    capacity = (1.2 * raw_ref["horizontal_mean"], 1.2 * raw_ref["vertical_mean"])
    theirs = session.rudy(pos, 64, 64, options.rudy_penalty_model, capacity=capacity, gradient=True)
    mine = backend.rudy(pos, options, capacity=capacity, gradient=True)
    for key in ("energy", "proxy_overflow", "maximum_utilization", "p95_utilization"):
        assert mine[key] == pytest.approx(theirs[key], rel=1e-6), key
    assert theirs["proxy_overflow"] > 0.0
    assert _rel(mine["gradient"], theirs["gradient"]) <= 1e-6
