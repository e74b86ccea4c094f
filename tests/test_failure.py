"""Failure detection without a GPU fault (needs a GPU).

* A field contraction's bounded wait runs out: the stall probe makes every
  contraction wait, for a bounded number of polls, on a barrier that nothing
  completes, before it issues any copy or takes tensor memory.  The evaluation
  must fail with MPGP_ERR_TIMEOUT (the error flag the host reads), the context
  must stay usable, and a new backend on the same layout must evaluate correctly.
* Non-finite host positions are refused with MPGP_ERR_NON_FINITE before anything
  is launched (CudaPlacementBackend.cu:945-948 refuses a non-finite result of
  the same evaluation), and the backend keeps working afterwards.
"""
from __future__ import annotations

import numpy as np
import pytest

import myplacement_b200 as mp
from myplacement_b200 import _abi
from myplacement_b200.design import Design

pytestmark = pytest.mark.gpu

STALL_POLLS = 1 << 12


def _golden_backend(golden_dir):
    g = np.load(golden_dir / "eval_small.npz")
    design = Design(**{k[4:]: g[k] for k in g.files if k.startswith("dsg_")}, name="eval_small")
    bins = int(g["bins"])
    layout = mp.build_layout(design, g["particle_width"], g["particle_height"], g["particle_layer"],
                             g["particle_pin_count"], int(g["movable_count"]), bins, bins, float(g["target_density"]),
                             g["static_fixed"], g["static_dark"])
    backend, reason = mp.try_create_backend(layout, 0)
    assert backend is not None, reason
    return g, layout, backend


def test_contraction_wait_runs_out_and_a_new_backend_recovers(gpu, golden_dir):
    g, layout, backend = _golden_backend(golden_dir)
    smoothing = float(g["smoothing"])
    backend.set_stall_probe(STALL_POLLS)
    for gradient in (True, False):
        with pytest.raises(mp.EngineError) as error:
            backend.evaluate(g["positions"], smoothing, gradient)
        assert error.value.status == _abi.MPGP_ERR_TIMEOUT
    backend.close()

    fresh, reason = mp.try_create_backend(layout, 0)
    assert fresh is not None, reason
    ev = fresh.evaluate(g["positions"], smoothing, True)
    assert ev["hpwl"] == pytest.approx(float(g["hpwl"]), rel=1e-5)
    assert ev["electrostatic_energy"] == pytest.approx(float(g["density_energy"]), rel=1e-5)
    scale = np.abs(g["density_gradient"]).max()
    assert np.abs(ev["density_gradient"] - g["density_gradient"]).max() <= 1e-4 * scale
    fresh.close()


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_non_finite_positions_are_refused(gpu, golden_dir, bad):
    g, _, backend = _golden_backend(golden_dir)
    positions = g["positions"].copy()
    positions[3, 1] = bad
    with pytest.raises(mp.EngineError) as error:
        backend.evaluate(positions, float(g["smoothing"]), True)
    assert error.value.status == _abi.MPGP_ERR_NON_FINITE
    ev = backend.evaluate(g["positions"], float(g["smoothing"]), True)
    assert ev["hpwl"] == pytest.approx(float(g["hpwl"]), rel=1e-5)
    backend.close()
