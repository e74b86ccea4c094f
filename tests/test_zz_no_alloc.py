"""The allocation-free wirelength entry point (needs a GPU).

mpgp_wirelength_noalloc serves callers that own all device memory and cannot
let the library allocate (a host framework whose allocator or fixed budget owns
the GPU, or a latency-critical loop that cannot afford cudaMalloc's implicit
synchronisation).  Its scratch is a fixed device array shared by every call, so
these tests call it several times in a row, on designs of different sizes, and
check every result: against mpgp_backend_evaluate at the same positions, and
against the reference CPU path (the oracle session's wire components).  The
tolerances are those of the parity suite: wire gradient within 1e-4 of the
largest component, smooth wirelength and HPWL within 1e-5 relative.  The file
is collected last and needs no state from other tests.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import myplacement_b200 as mp
from myplacement_b200 import _abi
from myplacement_b200.design import Design
from oracle.ref import default_options as ref_options

pytestmark = pytest.mark.gpu

GRADIENT_TOL = 1e-4
SCALAR_TOL = 1e-5
MAX_PINS = 1 << 20


def _golden_layout(golden_dir):
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


class NoAlloc:
    """Device copies of one layout and calls of mpgp_wirelength_noalloc on them."""

    def __init__(self, torch, layout, net_pin_start, net_weight, particle_count: int, net_count: int | None = None):
        self.torch = torch
        self.device = torch.device("cuda", 0)
        start, pins = _particle_csr(layout.pin_particle, particle_count)
        t = lambda a, dtype=None: torch.tensor(a, dtype=dtype, device=self.device)
        self.net_pin_start = t(np.asarray(net_pin_start).astype(np.int32))
        self.pin_particle = t(layout.pin_particle.astype(np.int32))
        self.pin_xy = t(np.stack([layout.pin_x, layout.pin_y], 1), torch.float64)
        self.net_weight = t(np.asarray(net_weight, np.float64), torch.float64)
        self.particle_pin_start = t(start)
        self.particle_pins = t(pins)
        self.particle_count = particle_count
        self.net_count = len(net_pin_start) - 1 if net_count is None else net_count
        self.pin_count = int(layout.pin_particle.shape[0])
        self.wire = torch.empty((particle_count, 2), dtype=torch.float64, device=self.device)
        self.totals = torch.empty(2, dtype=torch.float64, device=self.device)

    def __call__(self, positions: np.ndarray, smoothing: float):
        torch = self.torch
        lib = mp.load_library()
        stream = torch.cuda.current_stream(self.device)
        pos = torch.tensor(positions, dtype=torch.float64, device=self.device)
        status = lib.mpgp_wirelength_noalloc(
            pos.data_ptr(), self.net_pin_start.data_ptr(), self.pin_particle.data_ptr(), self.pin_xy.data_ptr(),
            self.net_weight.data_ptr(), self.net_count, self.pin_count, self.particle_pin_start.data_ptr(),
            self.particle_pins.data_ptr(), self.particle_count, smoothing, self.wire.data_ptr(),
            self.totals.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
        assert status == _abi.MPGP_OK, lib.mpgp_last_error()
        stream.synchronize()
        smooth, hpwl = self.totals.cpu().numpy()
        return self.wire.cpu().numpy().copy(), float(smooth), float(hpwl)


def _check(result, gradient, smooth, hpwl):
    mine, my_smooth, my_hpwl = result
    scale = np.abs(gradient).max()
    assert np.abs(mine - gradient).max() <= GRADIENT_TOL * scale
    assert my_smooth == pytest.approx(smooth, rel=SCALAR_TOL)
    assert my_hpwl == pytest.approx(hpwl, rel=SCALAR_TOL)


def test_noalloc_matches_backend_on_two_calls(gpu, golden_dir):
    torch = pytest.importorskip("torch")
    g, design, layout = _golden_layout(golden_dir)
    backend, reason = mp.try_create_backend(layout, 0)
    assert backend is not None, reason
    particles = g["positions"].shape[0]
    smoothing = float(g["smoothing"])
    rng = np.random.default_rng(4)
    placements = [g["positions"], g["positions"] + rng.normal(0.0, 15.0, g["positions"].shape)]
    expected = [backend.evaluate(p, smoothing, True) for p in placements]
    backend.close()
    call = NoAlloc(torch, layout, design.net_pin_start, design.net_weight, particles)
    results = [call(p, smoothing) for p in placements]  # two calls in a row through the shared scratch
    for result, reference in zip(results, expected):
        _check(result, reference["wire_gradient"], reference["smooth_wirelength"], reference["hpwl"])
    assert not np.array_equal(results[0][0], results[1][0])


def test_noalloc_matches_the_reference_session_on_many_nets(gpu, ref):
    """22k nets: more than the net pass's 2,048 blocks x 8 warps, so warps loop over nets;
    checked against the reference CPU path's wire components at identical positions."""
    torch = pytest.importorskip("torch")
    design, bins = mp.workload("mid_210k", scale=0.1)
    x, y = ref.random_placement(design, 2026)
    design = design.copy_with_positions(x, y)
    assert design.net_count > 2048 * 8
    session = ref.session(design, ref_options(bins_x=bins, bins_y=bins, target_density=0.9))
    layout = mp.build_layout(design, session.width, session.height, session.layer, session.pin_count,
                             session.movable_count, bins, bins, 0.9, *session.static_density())
    smoothing = 0.75 * max(design.core[2] - design.core[0], design.core[3] - design.core[1]) / bins
    call = NoAlloc(torch, layout, design.net_pin_start, design.net_weight, session.positions.shape[0])
    rng = np.random.default_rng(5)
    half = np.stack([session.width, session.height], 1) * 0.5
    low, high = np.array(design.core[:2]) + half, np.array(design.core[2:]) - half
    for trial in range(2):
        # Moved cells stay inside the core: the reference clamps centres to it first.
        positions = np.clip(session.positions + (rng.normal(0.0, 3.0, session.positions.shape) if trial else 0.0),
                            low, high)
        comp = session.components(positions, smoothing)
        _check(call(positions, smoothing), comp["wire_gradient"], comp["smooth_wirelength"], comp["hpwl"])


def test_noalloc_pins_outside_every_net_add_nothing(gpu, golden_dir, ref):
    """A call on a larger design fills the shared scratch; then a call on the small design
    with its last nets left out of net_pin_start, while their pins stay in the pin and
    particle lists, must equal the backend on the design without those nets."""
    torch = pytest.importorskip("torch")
    big, bins_big = mp.workload("mid_210k", scale=0.1)
    x, y = ref.random_placement(big, 7)
    big = big.copy_with_positions(x, y)
    session = ref.session(big, ref_options(bins_x=bins_big, bins_y=bins_big, target_density=0.9))
    big_layout = mp.build_layout(big, session.width, session.height, session.layer, session.pin_count,
                                 session.movable_count, bins_big, bins_big, 0.9, *session.static_density())
    big_call = NoAlloc(torch, big_layout, big.net_pin_start, big.net_weight, session.positions.shape[0])
    big_call(session.positions, 4.0)

    g, design, layout = _golden_layout(golden_dir)
    dropped = 40
    kept_nets = design.net_count - dropped
    kept_pins = int(design.net_pin_start[kept_nets])
    fields = {k: getattr(design, k) for k in design.__dataclass_fields__ if not k.startswith("_")}
    fields.update(net_weight=design.net_weight[:kept_nets], net_pin_start=design.net_pin_start[:kept_nets + 1],
                  pin_module=design.pin_module[:kept_pins], pin_offset_x=design.pin_offset_x[:kept_pins],
                  pin_offset_y=design.pin_offset_y[:kept_pins])
    fewer = Design(**fields)
    bins = int(g["bins"])
    fewer_layout = mp.build_layout(fewer, g["particle_width"], g["particle_height"], g["particle_layer"],
                                   g["particle_pin_count"], int(g["movable_count"]), bins, bins,
                                   float(g["target_density"]), g["static_fixed"], g["static_dark"])
    backend, reason = mp.try_create_backend(fewer_layout, 0)
    assert backend is not None, reason
    smoothing = float(g["smoothing"])
    expected = backend.evaluate(g["positions"], smoothing, True)
    backend.close()
    call = NoAlloc(torch, layout, design.net_pin_start, design.net_weight, g["positions"].shape[0],
                   net_count=kept_nets)
    assert call.pin_count > kept_pins
    for _ in range(2):
        _check(call(g["positions"], smoothing), expected["wire_gradient"], expected["smooth_wirelength"],
               expected["hpwl"])


def test_noalloc_rejects_inputs_beyond_its_scratch(gpu):
    lib = mp.load_library()
    status = lib.mpgp_wirelength_noalloc(None, None, None, None, None, 0, MAX_PINS + 1, None, None, 0, 1.0, None,
                                         None, None)
    assert status == _abi.MPGP_ERR_INVALID_ARGUMENT
    assert b"allocation-free limit" in lib.mpgp_last_error()
    # Exactly at the limit the size is accepted (the call then fails on its missing arrays instead).
    status = lib.mpgp_wirelength_noalloc(None, None, None, None, None, 0, MAX_PINS, None, None, 0, 1.0, None,
                                         None, None)
    assert status == _abi.MPGP_ERR_INVALID_ARGUMENT
    assert b"allocation-free limit" not in lib.mpgp_last_error()
