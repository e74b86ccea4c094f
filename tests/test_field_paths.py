"""The two field solves against the reference solver (needs a GPU).

The banded solve (one cluster per band of 64 spectral columns runs the forward DCT
and the inverse along y, then one contraction launch runs the inverse along x)
takes grids of up to 512 rows and 2,048 columns; by default only those taller
than 256 rows use it, and MPGP_FIELD_SOLVE=banded or =staged chooses for every
grid it takes.  The staged solve (four contraction launches) takes every grid.
Both must meet the field
tolerance against the reference's FP64 solver (ElectrostaticField::solveNeumann)
on grids that exercise every cluster shape of the banded solve -- one row block
(four CTAs of 16 columns), two (eight of 16), three (six of 32) and four (eight of
32) -- including non-square grids and widths that leave part of the last band
empty; and the two solves must agree with each other within twice that tolerance.
"""
from __future__ import annotations

import numpy as np
import pytest

import myplacement_b200 as mp
from oracle.ref import default_options as ref_options

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-5


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def _backend(ref, bins_x: int, bins_y: int):
    design, _ = mp.workload("small_5k")
    x, y = ref.random_placement(design, 2026)
    design = design.copy_with_positions(x, y)
    session = ref.session(design, ref_options(bins_x=bins_x, bins_y=bins_y, target_density=0.9))
    layout = mp.build_layout(design, session.width, session.height, session.layer, session.pin_count,
                             session.movable_count, bins_x, bins_y, 0.9, *session.static_density())
    backend, reason = mp.try_create_backend(layout, 0)
    assert backend is not None, reason
    return backend, design.core


@pytest.mark.parametrize("bins_x,bins_y", [(64, 64), (96, 128), (256, 256), (384, 320), (512, 512), (200, 448)])
def test_banded_and_staged_field_match_reference(gpu, ref, monkeypatch, bins_x, bins_y):
    rng = np.random.default_rng(bins_x * 1000 + bins_y)
    sources = [rng.standard_normal((bins_y, bins_x)) + 3.0, np.abs(rng.standard_normal((bins_y, bins_x))) ** 3]
    monkeypatch.setenv("MPGP_FIELD_SOLVE", "banded")
    banded, region = _backend(ref, bins_x, bins_y)
    monkeypatch.setenv("MPGP_FIELD_SOLVE", "staged")
    staged, _ = _backend(ref, bins_x, bins_y)
    monkeypatch.delenv("MPGP_FIELD_SOLVE")
    try:
        for source in sources:
            theirs = ref.field_solve(bins_x, bins_y, region, source)
            mine_banded = banded.field_solve(source)
            mine_staged = staged.field_solve(source)
            for a, s, b in zip(mine_banded, mine_staged, theirs):
                assert _rel(a, b) <= FIELD_TOL
                assert _rel(s, b) <= FIELD_TOL
                assert _rel(a, s) <= 2 * FIELD_TOL
    finally:
        banded.close()
        staged.close()
