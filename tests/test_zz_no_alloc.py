"""The allocation-free wirelength entry point against the regular backend (needs a GPU).

mpgp_wirelength_noalloc serves callers that own all device memory and cannot
let the library allocate (a host framework whose allocator or fixed budget owns
the GPU, or a latency-critical loop that cannot afford cudaMalloc's implicit
synchronisation).  Its scratch is a fixed device array shared by every call, so
this test calls it twice in a row at two different placements and checks each
result against mpgp_backend_evaluate at the same positions: wire gradient within
1e-4 of the largest component (the gradient tolerance of the parity suite),
smooth wirelength and HPWL within 1e-5 relative.  It lives in its own file,
collected last, and needs no state from other tests.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import myplacement_b200 as mp
from myplacement_b200 import _abi
from myplacement_b200.design import Design

pytestmark = pytest.mark.gpu

GRADIENT_TOL = 1e-4
SCALAR_TOL = 1e-5
MAX_PINS = 1 << 20


def _case(golden_dir):
    g = np.load(golden_dir / "eval_small.npz")
    design = Design(**{k[4:]: g[k] for k in g.files if k.startswith("dsg_")}, name="eval_small")
    bins = int(g["bins"])
    layout = mp.build_layout(design, g["particle_width"], g["particle_height"], g["particle_layer"],
                             g["particle_pin_count"], int(g["movable_count"]), bins, bins, float(g["target_density"]),
                             g["static_fixed"], g["static_dark"])
    return g, design, layout


def _particle_csr(pin_particle: np.ndarray, particle_count: int):
    movable = np.nonzero(pin_particle >= 0)[0]
    order = movable[np.argsort(pin_particle[movable], kind="stable")]
    counts = np.bincount(pin_particle[movable], minlength=particle_count)
    start = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return start, order.astype(np.int32)


def test_noalloc_matches_backend_on_two_calls(gpu, golden_dir):
    torch = pytest.importorskip("torch")
    g, design, layout = _case(golden_dir)
    backend, reason = mp.try_create_backend(layout, 0)
    assert backend is not None, reason
    particles = g["positions"].shape[0]
    smoothing = float(g["smoothing"])
    rng = np.random.default_rng(4)
    placements = [g["positions"], g["positions"] + rng.normal(0.0, 15.0, g["positions"].shape)]
    expected = [backend.evaluate(p, smoothing, True) for p in placements]
    backend.close()

    device = torch.device("cuda", 0)
    start, pins = _particle_csr(layout.pin_particle, particles)
    arrays = {
        "net_pin_start": torch.tensor(design.net_pin_start.astype(np.int32), device=device),
        "pin_particle": torch.tensor(layout.pin_particle.astype(np.int32), device=device),
        "pin_xy": torch.tensor(np.stack([layout.pin_x, layout.pin_y], 1), dtype=torch.float64, device=device),
        "net_weight": torch.tensor(design.net_weight, dtype=torch.float64, device=device),
        "particle_pin_start": torch.tensor(start, device=device),
        "particle_pins": torch.tensor(pins, device=device),
    }
    wire = torch.empty((particles, 2), dtype=torch.float64, device=device)
    totals = torch.empty(2, dtype=torch.float64, device=device)
    lib = mp.load_library()
    stream = torch.cuda.current_stream(device)
    results = []
    for positions in placements:  # two calls in a row through the shared scratch
        pos = torch.tensor(positions, dtype=torch.float64, device=device)
        status = lib.mpgp_wirelength_noalloc(
            pos.data_ptr(), arrays["net_pin_start"].data_ptr(), arrays["pin_particle"].data_ptr(),
            arrays["pin_xy"].data_ptr(), arrays["net_weight"].data_ptr(), design.net_count, design.pin_count,
            arrays["particle_pin_start"].data_ptr(), arrays["particle_pins"].data_ptr(), particles, smoothing,
            wire.data_ptr(), totals.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
        assert status == _abi.MPGP_OK, lib.mpgp_last_error()
        stream.synchronize()
        results.append((wire.cpu().numpy().copy(), totals.cpu().numpy().copy()))
    for (gradient, (smooth, hpwl)), reference in zip(results, expected):
        scale = np.abs(reference["wire_gradient"]).max()
        assert np.abs(gradient - reference["wire_gradient"]).max() <= GRADIENT_TOL * scale
        assert smooth == pytest.approx(reference["smooth_wirelength"], rel=SCALAR_TOL)
        assert hpwl == pytest.approx(reference["hpwl"], rel=SCALAR_TOL)
    assert not np.array_equal(results[0][0], results[1][0])


def test_noalloc_rejects_inputs_beyond_its_scratch(gpu):
    lib = mp.load_library()
    status = lib.mpgp_wirelength_noalloc(None, None, None, None, None, 0, MAX_PINS + 1, None, None, 0, 1.0, None,
                                         None, None)
    assert status == _abi.MPGP_ERR_INVALID_ARGUMENT
    assert b"allocation-free limit" in lib.mpgp_last_error()
