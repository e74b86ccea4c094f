"""ctypes access to the oracle libraries (test infrastructure only).

``ReferenceLibrary`` wraps ``oracle/_ref/libref_*.so`` -- the reference's own
global-placement code compiled by ``oracle/build_oracle.py`` -- and
``fixed_deposit`` wraps the project's fixed-point restatement in
``oracle/density_fixed.c``.  Only tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU baseline legs import this module.
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ORACLE = Path(__file__).resolve().parent
REPO = ORACLE.parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

from myplacement_b200 import _abi  # noqa: E402  (struct layouts shared with the product)

_d = C.POINTER(C.c_double)
_i32 = C.POINTER(C.c_int32)
_i64 = C.POINTER(C.c_int64)
_vp = C.c_void_p


def _ptr(array: np.ndarray | None, kind):
    return None if array is None else array.ctypes.data_as(kind)


class ReferenceFailure(RuntimeError):
    """An exception thrown by the reference code, as (status, message)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"reference status {status}: {message}")
        self.status = status
        self.message = message


class ReferenceLibrary:
    """One of libref_cpu.so / libref_cuda.so / libref_dropin.so."""

    def __init__(self, variant: str = "cpu"):
        path = ORACLE / "_ref" / f"libref_{variant}.so"
        if not path.is_file():
            raise FileNotFoundError(f"oracle library missing: {path} (run oracle/build_oracle.py)")
        self.path = path
        lib = C.CDLL(str(path))
        sig = {
            "ref_last_error": (C.c_char_p, []),
            "ref_random_placement": (C.c_int, [C.POINTER(_abi.Design), C.c_uint64, _d, _d]),
            "ref_global_place": (C.c_int, [C.POINTER(_abi.Design), C.POINTER(_abi.Options), _d, _d,
                                           C.POINTER(_abi.Result), C.POINTER(_abi.HistoryRow), C.c_int32]),
            "ref_session_create": (C.c_int, [C.POINTER(_abi.Design), C.POINTER(_abi.Options), C.POINTER(_vp)]),
            "ref_session_destroy": (None, [_vp]),
            "ref_session_counts": (C.c_int, [_vp, _i64, _i64, _i64]),
            "ref_session_particles": (C.c_int, [_vp, _d, _d, _d, _d, _i32, _i32]),
            "ref_session_static_density": (C.c_int, [_vp, _d, _d]),
            "ref_session_evaluate": (C.c_int, [_vp, _d, C.c_double, C.c_double, C.c_double, C.c_int, _d,
                                               C.POINTER(_abi.DensityMetrics), C.POINTER(_abi.DensityMetrics),
                                               _d, _d]),
            "ref_session_components": (C.c_int, [_vp, _d, C.c_double, _d, _d, _d, _d, _d, _d, _d, _d, _d, _d]),
            "ref_session_rudy": (C.c_int, [_vp, _d, C.c_int32, C.c_int32, C.c_double, C.c_int32, C.c_double,
                                           C.c_double, C.c_double, C.c_int, _d, _d]),
            "ref_field_solve": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                                          _d, _d, _d, _d]),
            "ref_field_sample": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                                           _d, C.c_int64, _d, _d]),
            "ref_density_map": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                          C.c_double, C.c_int32, _d, C.c_int32, _d, _i32, _d,
                                          C.POINTER(_abi.DensityMetrics)]),
            "ref_design_metrics": (C.c_int, [C.POINTER(_abi.Design), C.c_int32, C.c_int32, C.c_double, _d,
                                             C.POINTER(_abi.DensityMetrics)]),
            "ref_detailed_place": (C.c_int, [C.POINTER(_abi.Design), _i32, C.POINTER(_abi.DetailedOptions),
                                             C.c_int32, _d, _d, _i32, C.POINTER(_abi.DetailedResult)]),
            "ref_bookshelf_read": (C.c_int, [C.c_char_p, C.POINTER(_vp)]),
            "ref_bookshelf_destroy": (None, [_vp]),
            "ref_bookshelf_counts": (C.c_int, [_vp, _i64, _i64, _d]),
            "ref_bookshelf_modules": (C.c_int, [_vp, _d, _d, _d, _d, _i32, _i32, _i64, _i64]),
            "ref_bookshelf_nets": (C.c_int, [_vp, _d, _i64, _i64, _i32, _i64, _d, _d, _i32]),
            "ref_bookshelf_rows": (C.c_int, [_vp, _d, _d, _d, _d, _d, _i64, _i32]),
            "ref_bookshelf_module_name": (C.c_void_p, [_vp, C.c_int64, _i64]),
            "ref_bookshelf_net_name": (C.c_void_p, [_vp, C.c_int64, _i64]),
        }
        for name, (restype, argtypes) in sig.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        self.lib = lib

    def _check(self, status: int) -> None:
        if status != 0:
            raise RuntimeError(f"reference status {status}: {self.lib.ref_last_error().decode(errors='replace')}")

    # ---- whole runs -----------------------------------------------------------------
    def random_placement(self, design, seed: int) -> tuple[np.ndarray, np.ndarray]:
        x = np.empty(design.module_count)
        y = np.empty(design.module_count)
        s = design.as_c()
        self._check(self.lib.ref_random_placement(C.byref(s), seed, _ptr(x, _d), _ptr(y, _d)))
        return x, y

    def global_place(self, design, options: _abi.Options, history_capacity: int = 4096):
        x = design.module_x.copy()
        y = design.module_y.copy()
        result = _abi.Result()
        rows = (_abi.HistoryRow * history_capacity)()
        s = design.as_c()
        self._check(self.lib.ref_global_place(C.byref(s), C.byref(options), _ptr(x, _d), _ptr(y, _d),
                                              C.byref(result), rows, history_capacity))
        history = [rows[i].as_dict() for i in range(min(result.history_count, history_capacity))]
        return x, y, result, history

    def design_metrics(self, design, columns: int, rows: int, target_density: float):
        hpwl = C.c_double()
        metrics = _abi.DensityMetrics()
        s = design.as_c()
        self._check(self.lib.ref_design_metrics(C.byref(s), columns, rows, target_density, C.byref(hpwl),
                                                C.byref(metrics)))
        return hpwl.value, metrics.as_dict()

    # ---- single evaluations ------------------------------------------------------------
    def detailed_place(self, design, options: _abi.DetailedOptions, backend: int, row_orientation=None):
        """DetailedPlacer::run with `backend` (0 cpu, 1 cuda, 2 auto) of the linked
        backend; returns (x, y, orientation, result dict, backend used) or raises
        ReferenceFailure."""
        x = np.empty(design.module_count)
        y = np.empty(design.module_count)
        orientation = np.empty(design.module_count, np.int32)
        rows = None if row_orientation is None else np.ascontiguousarray(row_orientation, dtype=np.int32)
        result = _abi.DetailedResult()
        s = design.as_c()
        used = self.lib.ref_detailed_place(C.byref(s), _ptr(rows, _i32), C.byref(options), backend, _ptr(x, _d),
                                           _ptr(y, _d), _ptr(orientation, _i32), C.byref(result))
        if used < 0:
            raise ReferenceFailure(-used, self.lib.ref_last_error().decode(errors="replace"))
        return x, y, orientation, result.as_dict(), used

    def read_bookshelf(self, aux_path) -> dict:
        """BookshelfParser().parseAux(aux_path) of the linked reader, flattened.

        Raises ReferenceFailure with the status (MPGP_ERR_PARSE for ParseError)
        and the message when the reader throws."""
        lib = self.lib
        handle = _vp()
        status = lib.ref_bookshelf_read(str(aux_path).encode(), C.byref(handle))
        if status != 0:
            raise ReferenceFailure(status, lib.ref_last_error().decode(errors="replace"))
        try:
            counts = np.zeros(5, np.int64)
            declared = np.zeros(4, np.int64)
            regions = np.zeros(9)
            lib.ref_bookshelf_counts(handle, _ptr(counts, _i64), _ptr(declared, _i64), _ptr(regions, _d))
            modules, nets, pins, rows, movable = (int(c) for c in counts)
            out = {"declared": declared, "regions": regions, "movable_count": movable}
            f64 = lambda n: np.zeros(n)
            m = {k: f64(modules) for k in ("width", "height", "x", "y")}
            m["flags"] = np.zeros(modules, np.int32)
            m["orientation"] = np.zeros(modules, np.int32)
            m["pin_start"] = np.zeros(modules + 1, np.int64)
            m["pins"] = np.zeros(pins, np.int64)
            lib.ref_bookshelf_modules(handle, *(_ptr(m[k], _d) for k in ("width", "height", "x", "y")),
                                      _ptr(m["flags"], _i32), _ptr(m["orientation"], _i32),
                                      _ptr(m["pin_start"], _i64), _ptr(m["pins"], _i64))
            n = {"weight": f64(nets), "pin_start": np.zeros(nets + 1, np.int64), "pins": np.zeros(pins, np.int64),
                 "pin_module": np.zeros(pins, np.int32), "pin_net": np.zeros(pins, np.int64),
                 "offset_x": f64(pins), "offset_y": f64(pins), "direction": np.zeros(pins, np.int32)}
            lib.ref_bookshelf_nets(handle, _ptr(n["weight"], _d), _ptr(n["pin_start"], _i64), _ptr(n["pins"], _i64),
                                   _ptr(n["pin_module"], _i32), _ptr(n["pin_net"], _i64), _ptr(n["offset_x"], _d),
                                   _ptr(n["offset_y"], _d), _ptr(n["direction"], _i32))
            r = {k: f64(rows) for k in ("bottom", "height", "site_width", "site_spacing", "x_start")}
            r["site_count"] = np.zeros(rows, np.int64)
            r["orientation"] = np.zeros(rows, np.int32)
            lib.ref_bookshelf_rows(handle, *(_ptr(r[k], _d) for k in ("bottom", "height", "site_width",
                                                                      "site_spacing", "x_start")),
                                   _ptr(r["site_count"], _i64), _ptr(r["orientation"], _i32))
            out["modules"], out["nets"], out["rows"] = m, n, r
            length = C.c_int64()

            def name(fn, i):
                data = fn(handle, i, C.byref(length))
                return C.string_at(data, length.value).decode("utf-8", "surrogateescape") if length.value else ""

            out["module_names"] = [name(lib.ref_bookshelf_module_name, i) for i in range(modules)]
            out["net_names"] = [name(lib.ref_bookshelf_net_name, i) for i in range(nets)]
            return out
        finally:
            lib.ref_bookshelf_destroy(handle)

    def session(self, design, options: _abi.Options) -> "ReferenceSession":
        return ReferenceSession(self, design, options)

    def field_solve(self, columns: int, rows: int, region, deviation: np.ndarray):
        deviation = np.ascontiguousarray(deviation, dtype=np.float64).reshape(-1)
        out = [np.empty(columns * rows) for _ in range(3)]
        self._check(self.lib.ref_field_solve(columns, rows, *region, _ptr(deviation, _d),
                                             *(_ptr(a, _d) for a in out)))
        return [a.reshape(rows, columns) for a in out]

    def field_sample(self, columns: int, rows: int, region, deviation: np.ndarray, points: np.ndarray):
        deviation = np.ascontiguousarray(deviation, dtype=np.float64).reshape(-1)
        points = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
        out = np.empty_like(points)
        self._check(self.lib.ref_field_sample(columns, rows, *region, _ptr(deviation, _d), points.shape[0],
                                              _ptr(points, _d), _ptr(out, _d)))
        return out

    def density_map(self, region, columns: int, rows: int, target_density: float, placeable, rects, layers):
        placeable = np.ascontiguousarray(placeable, dtype=np.float64).reshape(-1, 4)
        rects = np.ascontiguousarray(rects, dtype=np.float64).reshape(-1, 4)
        layers = np.ascontiguousarray(layers, dtype=np.int32)
        bins = np.empty(columns * rows * 5)
        metrics = (_abi.DensityMetrics * 2)()
        self._check(self.lib.ref_density_map(*region, columns, rows, target_density, placeable.shape[0],
                                             _ptr(placeable, _d), rects.shape[0], _ptr(rects, _d),
                                             _ptr(layers, _i32), _ptr(bins, _d), metrics))
        return bins.reshape(rows, columns, 5), metrics[0].as_dict(), metrics[1].as_dict()


class ReferenceSession:
    """The reference's GlobalPlacementSession on the CPU path (one evaluation per call)."""

    def __init__(self, ref: ReferenceLibrary, design, options: _abi.Options):
        self.ref = ref
        self.design = design
        self.options = options
        self.handle = _vp()
        s = design.as_c()
        ref._check(ref.lib.ref_session_create(C.byref(s), C.byref(options), C.byref(self.handle)))
        particles, movable, fillers = C.c_int64(), C.c_int64(), C.c_int64()
        ref.lib.ref_session_counts(self.handle, C.byref(particles), C.byref(movable), C.byref(fillers))
        self.particle_count = particles.value
        self.movable_count = movable.value
        self.filler_count = fillers.value
        n = self.particle_count
        self.x, self.y, self.width, self.height = (np.empty(n) for _ in range(4))
        self.layer = np.empty(n, np.int32)
        self.pin_count = np.empty(n, np.int32)
        ref.lib.ref_session_particles(self.handle, _ptr(self.x, _d), _ptr(self.y, _d), _ptr(self.width, _d),
                                      _ptr(self.height, _d), _ptr(self.layer, _i32), _ptr(self.pin_count, _i32))

    def __del__(self):
        if getattr(self, "handle", None):
            self.ref.lib.ref_session_destroy(self.handle)
            self.handle = None

    @property
    def positions(self) -> np.ndarray:
        return np.stack([self.x, self.y], axis=1)

    def static_density(self):
        bins = self.options.bins_x * self.options.bins_y
        fixed, dark = np.empty(bins), np.empty(bins)
        self.ref.lib.ref_session_static_density(self.handle, _ptr(fixed, _d), _ptr(dark, _d))
        return fixed, dark

    def evaluate(self, positions: np.ndarray, smoothing: float, penalty: float, reference_penalty: float,
                 gradient: bool = True) -> dict:
        positions = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1)
        scalars = np.empty(8)
        optimizer, design = _abi.DensityMetrics(), _abi.DensityMetrics()
        raw = np.zeros(self.particle_count * 2)
        pre = np.zeros(self.particle_count * 2)
        self.ref._check(self.ref.lib.ref_session_evaluate(
            self.handle, _ptr(positions, _d), smoothing, penalty, reference_penalty, int(gradient),
            _ptr(scalars, _d), C.byref(optimizer), C.byref(design), _ptr(raw, _d), _ptr(pre, _d)))
        keys = ["hpwl", "smooth_wirelength", "density_energy", "objective", "wire_gradient_l1",
                "density_gradient_l1", "raw_gradient_norm", "preconditioned_gradient_norm"]
        out = dict(zip(keys, scalars.tolist()))
        out["optimizer_density"] = optimizer.as_dict()
        out["design_density"] = design.as_dict()
        out["raw_gradient"] = raw.reshape(-1, 2)
        out["preconditioned_gradient"] = pre.reshape(-1, 2)
        return out

    def components(self, positions: np.ndarray, smoothing: float) -> dict:
        positions = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1)
        n = self.particle_count
        bins = self.options.bins_x * self.options.bins_y
        wire_scalars = np.empty(2)
        wire = np.empty(2 * n)
        density = np.empty(2 * n)
        energy = C.c_double()
        layers = [np.empty(bins) for _ in range(3)]
        fields = [np.empty(bins) for _ in range(3)]
        self.ref._check(self.ref.lib.ref_session_components(
            self.handle, _ptr(positions, _d), smoothing, _ptr(wire_scalars, _d), _ptr(wire, _d),
            _ptr(density, _d), C.byref(energy), *(_ptr(a, _d) for a in layers), *(_ptr(a, _d) for a in fields)))
        shape = (self.options.bins_y, self.options.bins_x)
        return {
            "smooth_wirelength": wire_scalars[0], "hpwl": wire_scalars[1],
            "wire_gradient": wire.reshape(-1, 2), "density_gradient": density.reshape(-1, 2),
            "energy": energy.value,
            "movable": layers[0].reshape(shape), "macro": layers[1].reshape(shape),
            "filler": layers[2].reshape(shape),
            "potential": fields[0].reshape(shape), "field_x": fields[1].reshape(shape),
            "field_y": fields[2].reshape(shape),
        }

    def rudy(self, positions: np.ndarray, columns: int, rows: int, model: int, capacity=(0.0, 0.0),
             minimum_span: float = 0.25, temperature: float = 0.10, gradient: bool = False) -> dict:
        """evaluateRudy at `positions`: the ten metrics of RUDY_METRIC_NAMES and the per-particle subgradient."""
        positions = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1)
        metrics = np.empty(10)
        grad = np.zeros(positions.size)
        self.ref._check(self.ref.lib.ref_session_rudy(
            self.handle, _ptr(positions, _d), columns, rows, minimum_span, model, temperature, float(capacity[0]),
            float(capacity[1]), int(gradient), _ptr(metrics, _d), _ptr(grad, _d)))
        out = dict(zip(RUDY_METRIC_NAMES, metrics.tolist()))
        out["gradient"] = grad.reshape(-1, 2)
        return out


RUDY_METRIC_NAMES = ("horizontal_total", "vertical_total", "horizontal_mean", "vertical_mean", "horizontal_capacity",
                     "vertical_capacity", "proxy_overflow", "maximum_utilization", "p95_utilization", "energy")


# ---- the project's fixed-point restatement (oracle/density_fixed.c) ----------------------

_ORACLE_C: C.CDLL | None = None


def _oracle_c() -> C.CDLL:
    global _ORACLE_C
    if _ORACLE_C is None:
        path = ORACLE / "liboracle.so"
        if not path.is_file():
            raise FileNotFoundError(f"{path} missing (run oracle/build_oracle.py)")
        lib = C.CDLL(str(path))
        lib.oracle_deposit.restype = C.c_int
        lib.oracle_deposit.argtypes = [C.c_int64, _d, _d, _d, _d, _i32, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_int32, C.c_int32, _i64, _i64, _i64]
        lib.oracle_deposit_rects.restype = C.c_int
        lib.oracle_deposit_rects.argtypes = [C.c_int64, _d, C.c_double, C.c_double, C.c_double, C.c_double,
                                             C.c_int32, C.c_int32, _i64]
        _ORACLE_C = lib
    return _ORACLE_C


def fixed_deposit(x, y, width, height, layer, region, columns: int, rows: int):
    """Fixed-point movable/macro/filler layers (int64, units of bin_area * 2^-32)."""
    arrays = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, width, height)]
    layer = np.ascontiguousarray(layer, dtype=np.int32)
    out = [np.zeros(columns * rows, np.int64) for _ in range(3)]
    status = _oracle_c().oracle_deposit(arrays[0].shape[0], *(_ptr(a, _d) for a in arrays), _ptr(layer, _i32),
                                        *region, columns, rows, *(_ptr(a, _i64) for a in out))
    if status != 0:
        raise ValueError("oracle_deposit rejected its arguments")
    return [a.reshape(rows, columns) for a in out]


def fixed_deposit_rects(rects, region, columns: int, rows: int):
    rects = np.ascontiguousarray(rects, dtype=np.float64).reshape(-1, 4)
    out = np.zeros(columns * rows, np.int64)
    status = _oracle_c().oracle_deposit_rects(rects.shape[0], _ptr(rects, _d), *region, columns, rows,
                                              _ptr(out, _i64))
    if status != 0:
        raise ValueError("oracle_deposit_rects rejected its arguments")
    return out.reshape(rows, columns)


def default_options(**overrides) -> _abi.Options:
    """GlobalPlacementOptions defaults (include/myplacement/placement/GlobalPlacer.hpp:26-80)."""
    o = _abi.Options()
    o.iterations, o.bins_x, o.bins_y, o.report_interval = 280, 64, 64, 10
    o.target_density, o.maximum_bin_overflow = 0.85, 0.10
    o.initial_smoothing, o.final_smoothing = 0.75, 0.12
    o.maximum_movement_in_bins, o.penalty_growth = 0.22, 1.035
    o.optimizer, o.maximum_backtracks = 1, 6
    o.backtracking_ratio, o.armijo_coefficient, o.maximum_momentum = 0.5, 1e-4, 0.92
    o.initial_movement_in_bins, o.objective_increase_for_density = 0.12, 0.002
    o.hpwl_growth_restart_threshold, o.density_stall_threshold = 0.02, 0.002
    o.density_penalty_increase, o.density_penalty_decrease = 1.05, 0.88
    o.minimum_density_penalty, o.maximum_density_penalty = 1e-4, 1e6
    o.smoothing_overflow_exponent, o.feasible_refinement_iterations = 1.0, 12
    o.maximum_fillers, o.seed = 50_000, 2026
    o.rudy_columns, o.rudy_rows = 64, 64
    o.rudy_minimum_span_in_bins, o.rudy_capacity_factor, o.rudy_softplus_temperature = 0.25, 1.0, 0.10
    o.rudy_penalty_model, o.rudy_validation_bins, o.rudy_validation_capacity_factor = 0, 0, 1.50
    o.routability_start_overflow, o.routability_weight_scale, o.routability_ramp_iterations = 0.20, 0.20, 24
    o.density_field_boundary, o.compute_backend, o.cuda_device = 1, 0, 1
    o.maximum_cuda_memory_bytes = 40 * 1024 ** 3
    for key, value in overrides.items():
        setattr(o, key, value)
    return o
