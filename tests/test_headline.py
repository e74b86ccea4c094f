"""Parity on the headline configuration at full size (needs a GPU): the mid design
of 210,000 cells, 400 fixed macros, 1,200 terminals, 220,000 nets (~848k pins),
512 x 512 bins, target density 0.9 -- the configuration the bench line is quoted on.

Against the reference CPU path (FP64, oracle/_ref/libref_cpu.so) at identical positions,
at the random initial placement and at a spread placement 60 iterations into a run:
  * the three density layers bit-exact against the fixed-point oracle;
  * HPWL, smooth wirelength, density energy and all sixteen DensityMetrics values
    within 1e-5 relative;
  * wire and density gradients within 1e-4 * max |g_ref|;
and the Neumann field (potential, Ex, Ey) of the design's own density deviation and
of a heavy-tailed random source within 1e-5 * max |E_ref|.
"""
from __future__ import annotations

import numpy as np
import pytest

import myplacement_b200 as mp
from oracle.ref import default_options as ref_options, fixed_deposit

pytestmark = pytest.mark.gpu

SCALAR_TOL = 1e-5
GRADIENT_TOL = 1e-4
FIELD_TOL = 1e-5


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.fixture(scope="module")
def headline(ref):
    design, bins = mp.workload("mid_210k")
    x, y = ref.random_placement(design, 2026)
    design = design.copy_with_positions(x, y)
    assert bins == 512 and design.net_count == 220_000
    session = ref.session(design, ref_options(bins_x=bins, bins_y=bins, target_density=0.9))
    layout = mp.build_layout(design, session.width, session.height, session.layer, session.pin_count,
                             session.movable_count, bins, bins, 0.9, *session.static_density())
    backend, reason = mp.try_create_backend(layout, 0)
    assert backend is not None, reason
    # A spread placement: the engine's own run, 60 iterations in (early stop off).
    spread = mp.GlobalPlacer().run(design, mp.default_options(bins_x=bins, bins_y=bins, target_density=0.9,
                                                              iterations=60,
                                                              feasible_refinement_iterations=10 ** 9))
    movable = design.movable_mask
    later = session.positions.copy()
    later[:session.movable_count, 0] = spread.module_x[movable]
    later[:session.movable_count, 1] = spread.module_y[movable]
    yield design, bins, session, backend, {"initial": session.positions, "spread": later}
    backend.close()


@pytest.mark.parametrize("placement", ["initial", "spread"])
def test_headline_evaluation_matches_reference(gpu, headline, placement):
    design, bins, session, backend, placements = headline
    pos = placements[placement]
    smoothing = 0.75 * max(design.core[2] - design.core[0], design.core[3] - design.core[1]) / bins
    comp = session.components(pos, smoothing)
    full = session.evaluate(pos, smoothing, 0.5, 0.5, True)
    ev = backend.evaluate(pos, smoothing, True)
    assert ev["hpwl"] == pytest.approx(comp["hpwl"], rel=SCALAR_TOL)
    assert ev["smooth_wirelength"] == pytest.approx(comp["smooth_wirelength"], rel=SCALAR_TOL)
    assert ev["electrostatic_energy"] == pytest.approx(comp["energy"], rel=SCALAR_TOL)
    for key in ("optimizer_density", "design_density"):
        mine = np.array([ev[key][k] for k in mp._abi.DENSITY_METRIC_FIELDS])
        theirs = np.array([full[key][k] for k in mp._abi.DENSITY_METRIC_FIELDS])
        np.testing.assert_allclose(mine, theirs, rtol=SCALAR_TOL, atol=1e-9, err_msg=key)
    assert _rel(ev["wire_gradient"], comp["wire_gradient"]) <= GRADIENT_TOL
    assert _rel(ev["density_gradient"], comp["density_gradient"]) <= GRADIENT_TOL
    layers = backend.density_layers(bins, bins)
    expected = fixed_deposit(pos[:, 0], pos[:, 1], session.width, session.height, session.layer, design.core,
                             bins, bins)
    for mine, theirs in zip(layers, expected):
        assert np.array_equal(mine, theirs)


def test_headline_field_matches_reference(gpu, ref, headline):
    design, bins, session, backend, placements = headline
    comp = session.components(placements["spread"], 4.0)
    target = 0.9
    bin_area = (design.core[2] - design.core[0]) * (design.core[3] - design.core[1]) / (bins * bins)
    fixed, dark = session.static_density()
    charge = (comp["movable"].reshape(-1) + target * (comp["macro"] + comp["filler"]).reshape(-1)
              + target * (fixed + dark))
    deviation = (charge / bin_area - target).reshape(bins, bins)
    rng = np.random.default_rng(6)
    for source in (deviation, np.abs(rng.standard_normal((bins, bins))) ** 3):
        mine = backend.field_solve(source)
        theirs = ref.field_solve(bins, bins, design.core, source)
        for a, b in zip(mine, theirs):
            assert _rel(a, b) <= FIELD_TOL
