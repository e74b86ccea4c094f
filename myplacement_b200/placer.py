"""Python mirror of the reference's global-placement API over libmpgp.so.

``GlobalPlacer().run(design, options)`` mirrors ``myplacement::GlobalPlacer::run``
(include/myplacement/placement/GlobalPlacer.hpp:131-134) for
``compute_backend = cuda``: the same options, result fields and history rows.
``CudaPlacementBackend`` mirrors ``myplacement::detail::CudaPlacementBackend``
(src/placement/CudaPlacementBackend.hpp:25-39) -- one evaluation per call with
host positions -- and ``try_create_backend`` mirrors
``tryCreateCudaPlacementBackend`` (returns ``(None, reason)`` on a recoverable
failure).  Everything here is a thin wrapper: the work is in the native engine.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import check, load_library
from .design import Design

_d = C.POINTER(C.c_double)
_i32 = C.POINTER(C.c_int32)
_i64 = C.POINTER(C.c_int64)


def _ptr(array, kind):
    return None if array is None else array.ctypes.data_as(kind)


def default_options(**overrides) -> _abi.Options:
    """GlobalPlacementOptions defaults (GlobalPlacer.hpp:26-80), compute backend cuda on device 0."""
    options = _abi.Options()
    load_library().mpgp_options_default(C.byref(options))
    for key, value in overrides.items():
        if not hasattr(options, key):
            raise AttributeError(f"unknown option {key}")
        setattr(options, key, value)
    return options


@dataclass
class PlacementResult:
    """GlobalPlacementResult (GlobalPlacer.hpp:107-129) plus the placed module centres."""

    module_x: np.ndarray
    module_y: np.ndarray
    result: dict
    history: list[dict] = field(default_factory=list)

    def __getattr__(self, name):
        result = self.__dict__.get("result")
        if result is not None and name in result:
            return result[name]
        raise AttributeError(name)


def random_placement(design: Design, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """randomPlacement (InitialPlacer.cpp:102-121): movable centres uniform in the core."""
    lib = load_library()
    x = np.empty(design.module_count)
    y = np.empty(design.module_count)
    s = design.as_c()
    check(lib.mpgp_random_placement(C.byref(s), seed, _ptr(x, _d), _ptr(y, _d)))
    return x, y


class GlobalPlacer:
    """GlobalPlacer::run for the adaptive optimizer on the B200 engine."""

    def run(self, design: Design, options: _abi.Options, history_capacity: int | None = None) -> PlacementResult:
        lib = load_library()
        capacity = history_capacity if history_capacity is not None else max(1, options.iterations)
        x = design.module_x.copy()
        y = design.module_y.copy()
        result = _abi.Result()
        rows = (_abi.HistoryRow * capacity)()
        s = design.as_c()
        check(lib.mpgp_global_place(C.byref(s), C.byref(options), _ptr(x, _d), _ptr(y, _d), C.byref(result), rows,
                                    capacity))
        history = [rows[i].as_dict() for i in range(min(result.history_count, capacity))]
        return PlacementResult(x, y, result.as_dict(), history)


class Session:
    """A global-placement run split into steps (mpgp_session_*)."""

    def __init__(self, design: Design, options: _abi.Options):
        self.lib = load_library()
        self.design = design
        self.options = options
        self._design_c = design.as_c()
        self.handle = C.c_void_p()
        check(self.lib.mpgp_session_create(C.byref(self._design_c), C.byref(options), C.byref(self.handle)))

    def step(self, iterations: int) -> tuple[int, bool]:
        completed = C.c_int32()
        done = C.c_int32()
        check(self.lib.mpgp_session_step(self.handle, iterations, C.byref(completed), C.byref(done)))
        return completed.value, bool(done.value)

    def finish(self, history_capacity: int | None = None) -> PlacementResult:
        capacity = history_capacity if history_capacity is not None else max(1, self.options.iterations)
        x = np.empty(self.design.module_count)
        y = np.empty(self.design.module_count)
        result = _abi.Result()
        rows = (_abi.HistoryRow * capacity)()
        check(self.lib.mpgp_session_finish(self.handle, _ptr(x, _d), _ptr(y, _d), C.byref(result), rows, capacity))
        history = [rows[i].as_dict() for i in range(min(result.history_count, capacity))]
        return PlacementResult(x, y, result.as_dict(), history)

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.mpgp_session_kernel_launches(self.handle))

    @property
    def stream(self) -> int:
        return int(self.lib.mpgp_session_stream(self.handle) or 0)

    def set_profiling(self, families=True) -> None:
        """Times every launch of the given kernel families (names, or True for all, False for none)."""
        if families is True:
            mask = (1 << self.lib.mpgp_kernel_kind_count()) - 1
        elif families is False or families is None:
            mask = 0
        else:
            names = [self.lib.mpgp_kernel_kind_name(k).decode() for k in range(self.lib.mpgp_kernel_kind_count())]
            mask = 0
            for name in families:
                mask |= 1 << names.index(name)
        check(self.lib.mpgp_session_set_profiling(self.handle, mask))

    def reset_kernel_stats(self) -> None:
        check(self.lib.mpgp_session_reset_kernel_stats(self.handle))

    def kernel_stats(self) -> dict:
        """{family: (launches, device milliseconds)} accumulated while profiling was on."""
        n = self.lib.mpgp_kernel_kind_count()
        launches = np.zeros(n, np.int64)
        ms = np.zeros(n)
        check(self.lib.mpgp_session_kernel_stats(self.handle, _ptr(launches, _i64), _ptr(ms, _d), n))
        return {self.lib.mpgp_kernel_kind_name(k).decode(): (int(launches[k]), float(ms[k])) for k in range(n)}

    def transfer_bytes(self) -> tuple[int, int]:
        to_device, to_host = C.c_uint64(), C.c_uint64()
        check(self.lib.mpgp_session_transfer_bytes(self.handle, C.byref(to_device), C.byref(to_host)))
        return int(to_device.value), int(to_host.value)

    def positions(self, particle_count: int) -> np.ndarray:
        xy = np.empty(2 * particle_count)
        check(self.lib.mpgp_session_positions(self.handle, _ptr(xy, _d)))
        return xy.reshape(-1, 2)

    def close(self) -> None:
        if self.handle:
            self.lib.mpgp_session_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def host_setup(design: Design, options: _abi.Options) -> dict:
    """The host session setup (fillers, static density, preconditioner); needs no GPU."""
    lib = load_library()
    s = design.as_c()
    handle = C.c_void_p()
    check(lib.mpgp_setup_create(C.byref(s), C.byref(options), C.byref(handle)))
    try:
        n, m = C.c_int64(), C.c_int64()
        check(lib.mpgp_setup_particles(handle, C.byref(n), C.byref(m), None, None, None, None, None, None))
        count = n.value
        out = {k: np.empty(count) for k in ("x", "y", "width", "height", "preconditioner")}
        out["layer"] = np.empty(count, np.int32)
        check(lib.mpgp_setup_particles(handle, C.byref(n), C.byref(m), _ptr(out["x"], _d), _ptr(out["y"], _d),
                                       _ptr(out["width"], _d), _ptr(out["height"], _d), _ptr(out["layer"], _i32),
                                       _ptr(out["preconditioner"], _d)))
        bins = options.bins_x * options.bins_y
        out["static_fixed"], out["static_dark"] = np.empty(bins), np.empty(bins)
        check(lib.mpgp_setup_static_density(handle, _ptr(out["static_fixed"], _d), _ptr(out["static_dark"], _d)))
        out["particle_count"] = count
        out["movable_count"] = m.value
        return out
    finally:
        lib.mpgp_setup_destroy(handle)


@dataclass
class BackendLayout:
    """The flattened inputs of tryCreateCudaPlacementBackend (buildHostLayout, CudaPlacementBackend.cu:784-839)."""

    particle_width: np.ndarray
    particle_height: np.ndarray
    particle_layer: np.ndarray
    particle_pin_count: np.ndarray
    movable_count: int
    net_weight: np.ndarray
    net_pin_start: np.ndarray
    pin_particle: np.ndarray
    pin_x: np.ndarray
    pin_y: np.ndarray
    bins_x: int
    bins_y: int
    region: tuple[float, float, float, float]
    target_density: float
    static_fixed: np.ndarray
    static_dark: np.ndarray

    def as_c(self) -> _abi.Layout:
        f64 = lambda a: np.ascontiguousarray(a, np.float64)
        i32 = lambda a: np.ascontiguousarray(a, np.int32)
        i64 = lambda a: np.ascontiguousarray(a, np.int64)
        self._keep = [f64(self.particle_width), f64(self.particle_height), i32(self.particle_layer),
                      i32(self.particle_pin_count), f64(self.net_weight), i64(self.net_pin_start),
                      i32(self.pin_particle), f64(self.pin_x), f64(self.pin_y), f64(self.static_fixed),
                      f64(self.static_dark)]
        k = self._keep
        s = _abi.Layout()
        s.particle_count = k[0].shape[0]
        s.movable_count = self.movable_count
        s.particle_width, s.particle_height = _ptr(k[0], _d), _ptr(k[1], _d)
        s.particle_layer, s.particle_pin_count = _ptr(k[2], _i32), _ptr(k[3], _i32)
        s.net_count = k[4].shape[0]
        s.net_weight, s.net_pin_start = _ptr(k[4], _d), _ptr(k[5], _i64)
        s.pin_count = k[6].shape[0]
        s.pin_particle, s.pin_x, s.pin_y = _ptr(k[6], _i32), _ptr(k[7], _d), _ptr(k[8], _d)
        s.bins_x, s.bins_y = self.bins_x, self.bins_y
        s.region_llx, s.region_lly, s.region_urx, s.region_ury = self.region
        s.target_density = self.target_density
        s.static_fixed_area, s.static_dark_area = _ptr(k[9], _d), _ptr(k[10], _d)
        return s


def build_layout(design: Design, particle_width, particle_height, particle_layer, particle_pin_count,
                 movable_count: int, bins_x: int, bins_y: int, target_density: float, static_fixed,
                 static_dark) -> BackendLayout:
    """buildHostLayout (CudaPlacementBackend.cu:784-839) for designs whose orientation is North."""
    movable = np.nonzero(design.movable_mask)[0]
    module_particle = np.full(design.module_count, -1, np.int32)
    module_particle[movable] = np.arange(movable.shape[0], dtype=np.int32)
    pin_particle = module_particle[design.pin_module]
    static = pin_particle < 0
    pin_x = design.pin_offset_x.copy()
    pin_y = design.pin_offset_y.copy()
    pin_x[static] = design.module_x[design.pin_module[static]] + design.pin_offset_x[static]
    pin_y[static] = design.module_y[design.pin_module[static]] + design.pin_offset_y[static]
    return BackendLayout(particle_width, particle_height, particle_layer, particle_pin_count, movable_count,
                         design.net_weight, design.net_pin_start, pin_particle, pin_x, pin_y, bins_x, bins_y,
                         design.core, target_density, static_fixed, static_dark)


RUDY_METRIC_NAMES = ("horizontal_total", "vertical_total", "horizontal_mean", "vertical_mean", "horizontal_capacity",
                     "vertical_capacity", "proxy_overflow", "maximum_utilization", "p95_utilization", "energy")


class CudaPlacementBackend:
    """CudaPlacementBackend::evaluate over mpgp_backend_* (host positions in, host gradients out)."""

    def __init__(self, handle: C.c_void_p, particle_count: int):
        self.lib = load_library()
        self.handle = handle
        self.particle_count = particle_count

    def evaluate(self, positions: np.ndarray, smoothing: float, calculate_gradient: bool = True) -> dict:
        positions = np.ascontiguousarray(positions, np.float64).reshape(-1)
        if positions.shape[0] != 2 * self.particle_count:
            raise ValueError("CUDA placement positions do not match the particle count.")
        out = _abi.Evaluation()
        wire = np.zeros(2 * self.particle_count)
        density = np.zeros(2 * self.particle_count)
        check(self.lib.mpgp_backend_evaluate(self.handle, _ptr(positions, _d), smoothing, int(calculate_gradient),
                                             C.byref(out), _ptr(wire, _d), _ptr(density, _d)))
        result = {
            "hpwl": out.hpwl, "smooth_wirelength": out.smooth_wirelength,
            "electrostatic_energy": out.electrostatic_energy,
            "optimizer_density": out.optimizer_density.as_dict(), "design_density": out.design_density.as_dict(),
        }
        if calculate_gradient:
            result["wire_gradient"] = wire.reshape(-1, 2)
            result["density_gradient"] = density.reshape(-1, 2)
        return result

    def set_stall_probe(self, polls: int) -> None:
        """Failure-detection hook: later field contractions wait out a barrier nothing completes."""
        check(self.lib.mpgp_backend_set_stall_probe(self.handle, int(polls)))

    def density_layers(self, bins_x: int, bins_y: int):
        """The fixed-point layers (movable, macro, filler) of the last evaluated positions."""
        out = [np.empty(bins_x * bins_y, np.int64) for _ in range(3)]
        check(self.lib.mpgp_backend_density_layers(self.handle, *(_ptr(a, _i64) for a in out)))
        return [a.reshape(bins_y, bins_x) for a in out]

    def field_solve(self, deviation: np.ndarray):
        deviation = np.ascontiguousarray(deviation, np.float64)
        out = [np.empty(deviation.size) for _ in range(3)]
        check(self.lib.mpgp_backend_field_solve(self.handle, _ptr(deviation.reshape(-1), _d),
                                                *(_ptr(a, _d) for a in out)))
        return [a.reshape(deviation.shape) for a in out]

    def rudy(self, positions: np.ndarray, options, capacity=(0.0, 0.0), gradient: bool = False) -> dict:
        """The RUDY metrics (and subgradient) of one placement on the backend's nets.

        `options` supplies the grid, minimum span, penalty model and softplus
        temperature; the first call fixes the grid.  The ten metrics are named
        by RUDY_METRIC_NAMES; with `gradient` the result also holds the
        per-particle subgradient and the energy of the evaluation that made it.
        """
        positions = np.ascontiguousarray(positions, np.float64).reshape(-1)
        metrics = np.empty(10)
        energy = C.c_double(0.0)
        grad = np.zeros(positions.size)
        check(self.lib.mpgp_backend_rudy(self.handle, C.byref(options), _ptr(positions, _d), float(capacity[0]),
                                         float(capacity[1]), int(gradient), _ptr(metrics, _d), C.byref(energy),
                                         _ptr(grad, _d)))
        out = dict(zip(RUDY_METRIC_NAMES, metrics.tolist()))
        if gradient:
            out["gradient"] = grad.reshape(-1, 2)
            out["evaluation_energy"] = energy.value
        return out

    def device(self) -> int:
        return int(self.lib.mpgp_backend_device(self.handle))

    def reserved_bytes(self) -> int:
        return int(self.lib.mpgp_backend_reserved_bytes(self.handle))

    def close(self) -> None:
        if self.handle:
            self.lib.mpgp_backend_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def try_create_backend(layout: BackendLayout, device: int = 0, maximum_bytes: int = 40 * 1024 ** 3):
    """tryCreateCudaPlacementBackend: (backend, "") or (None, reason)."""
    lib = load_library()
    s = layout.as_c()
    handle = C.c_void_p()
    reason = C.create_string_buffer(512)
    status = lib.mpgp_backend_create(C.byref(s), device, maximum_bytes, C.byref(handle), reason, 512)
    if status == _abi.MPGP_ERR_UNAVAILABLE:
        return None, reason.value.decode(errors="replace")
    check(status)
    return CudaPlacementBackend(handle, int(s.particle_count)), ""


# ---- batched and served forms ------------------------------------------------------


def estimate_bytes(design: Design, options: _abi.Options) -> int:
    """Upper bound of the device bytes one placement of `design` reserves (the server's admission unit)."""
    lib = load_library()
    out = C.c_uint64()
    s = design.as_c()
    check(lib.mpgp_estimate_bytes(C.byref(s), C.byref(options), C.byref(out)))
    return int(out.value)


class PlacementServer:
    """Many placements at once on one GPU (mpgp_server_*): submit jobs as they arrive, take results.

    Each job is a full adaptive global placement (GlobalPlacer.run).  `workers`
    host threads each drive one device-resident session; a job starts when a
    worker is free and its estimated footprint fits in `memory_budget` (bytes;
    0 = 90 % of the device's free memory).  With `batched` the running jobs'
    evaluations share batched launches (one per kernel family and round);
    otherwise every job launches its own kernels.  Results do not depend on the
    mix or the mode.
    """

    def __init__(self, device: int = 0, memory_budget: int = 0, workers: int = 8, batched: bool = True):
        self.lib = load_library()
        self.handle = C.c_void_p()
        check(self.lib.mpgp_server_create_mode(device, memory_budget, workers, int(batched), C.byref(self.handle)))
        self._modules: dict[int, int] = {}
        self._capacity: dict[int, int] = {}

    def submit(self, design: Design, options: _abi.Options) -> int:
        job = C.c_int64()
        s = design.as_c()
        check(self.lib.mpgp_server_submit(self.handle, C.byref(s), C.byref(options), C.byref(job)))
        self._modules[job.value] = design.module_count
        self._capacity[job.value] = max(1, options.iterations)
        return int(job.value)

    def wait(self, job: int, timeout: float = -1.0) -> bool:
        done = C.c_int32()
        check(self.lib.mpgp_server_wait(self.handle, job, timeout, C.byref(done)))
        return bool(done.value)

    def take(self, job: int, history: bool = True) -> tuple[PlacementResult, dict]:
        """The finished job's PlacementResult and its timing (queued, run, latency seconds; footprint)."""
        n = self._modules.pop(job)
        capacity = self._capacity.pop(job) if history else 0
        x, y = np.empty(n), np.empty(n)
        result = _abi.Result()
        stats = _abi.JobStats()
        rows = (_abi.HistoryRow * max(1, capacity))()
        check(self.lib.mpgp_server_take(self.handle, job, _ptr(x, _d), _ptr(y, _d), C.byref(result), rows, capacity,
                                        C.byref(stats)))
        rows_kept = [rows[i].as_dict() for i in range(min(result.history_count, capacity))]
        return PlacementResult(x, y, result.as_dict(), rows_kept), stats.as_dict()

    def stats(self) -> dict:
        out = _abi.ServerStats()
        check(self.lib.mpgp_server_stats_get(self.handle, C.byref(out)))
        return out.as_dict()

    def close(self) -> None:
        if self.handle:
            self.lib.mpgp_server_destroy(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()


def batch_place(designs: list[Design], options: list[_abi.Options], device: int = 0, workers: int = 16,
                memory_budget: int = 0, batched: bool = True) -> tuple[list[PlacementResult], list[dict], dict]:
    """The batched form (mpgp_batch_place): every design placed, many at once (with `batched`, in shared
    batched launches); (results, job stats, server stats)."""
    lib = load_library()
    count = len(designs)
    structs = (_abi.Design * count)(*[d.as_c() for d in designs])
    opts = (_abi.Options * count)(*options)
    xs = [np.empty(d.module_count) for d in designs]
    ys = [np.empty(d.module_count) for d in designs]
    px = (_d * count)(*[_ptr(a, _d) for a in xs])
    py = (_d * count)(*[_ptr(a, _d) for a in ys])
    results = (_abi.Result * count)()
    job_stats = (_abi.JobStats * count)()
    server_stats = _abi.ServerStats()
    check(lib.mpgp_batch_place(count, structs, opts, device, workers, int(batched), memory_budget, px, py, results,
                               job_stats, C.byref(server_stats)))
    placed = [PlacementResult(xs[i], ys[i], results[i].as_dict()) for i in range(count)]
    return placed, [job_stats[i].as_dict() for i in range(count)], server_stats.as_dict()
