"""ctypes mirror of include/mpgp.h and the loader of libmpgp.so.

The engine is the native library; this module only declares its structs and
function signatures.  Loading fails loudly when the library has not been built:
there is no Python or CPU fallback for the engine.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
LIBRARY_PATH = PACKAGE_DIR / "libmpgp.so"

MPGP_OK = 0
MPGP_ERR_INVALID_ARGUMENT = 1
MPGP_ERR_RUNTIME = 2
MPGP_ERR_CUDA = 3
MPGP_ERR_BUDGET = 4
MPGP_ERR_NON_FINITE = 5
MPGP_ERR_UNAVAILABLE = 6
MPGP_ERR_TIMEOUT = 7
MPGP_ERR_PARSE = 8

MODULE_TERMINAL = 1
MODULE_FIXED = 2
LAYER_STANDARD, LAYER_MACRO, LAYER_FILLER = 0, 1, 2
BACKEND_CPU, BACKEND_CUDA, BACKEND_AUTO = 0, 1, 2
RUDY_DISABLED, RUDY_HINGE_L2, RUDY_SOFTPLUS_L2, RUDY_HINGE_L4 = 0, 1, 2, 3

_d = C.POINTER(C.c_double)
_i32 = C.POINTER(C.c_int32)
_i64 = C.POINTER(C.c_int64)


class Design(C.Structure):
    _fields_ = [
        ("module_count", C.c_int32),
        ("module_width", _d),
        ("module_height", _d),
        ("module_x", _d),
        ("module_y", _d),
        ("module_flags", _i32),
        ("module_orientation", _i32),
        ("net_count", C.c_int32),
        ("net_weight", _d),
        ("net_pin_start", _i64),
        ("pin_count", C.c_int64),
        ("pin_module", _i32),
        ("pin_offset_x", _d),
        ("pin_offset_y", _d),
        ("row_count", C.c_int32),
        ("row_bottom", _d),
        ("row_height", _d),
        ("row_site_width", _d),
        ("row_site_spacing", _d),
        ("row_x_start", _d),
        ("row_site_count", _i64),
    ]


DETAILED_NONE, DETAILED_ADJACENT_SWAP, DETAILED_WINDOW_REORDER = 0, 1, 2


class DetailedOptions(C.Structure):
    _fields_ = [
        ("method", C.c_int32),
        ("passes", C.c_int32),
        ("window_size", C.c_int32),
        ("cuda_device", C.c_int32),
        ("maximum_net_degree", C.c_uint64),
        ("improvement_epsilon", C.c_double),
        ("maximum_cuda_memory_bytes", C.c_uint64),
    ]


class DetailedResult(C.Structure):
    _fields_ = [
        ("hpwl_before", C.c_double),
        ("hpwl_after", C.c_double),
        ("elapsed_seconds", C.c_double),
        ("evaluated_windows", C.c_uint64),
        ("evaluated_permutations", C.c_uint64),
        ("accepted_operations", C.c_uint64),
        ("completed_passes", C.c_int32),
        ("cuda_device_used", C.c_int32),
        ("cuda_reserved_memory_bytes", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class BookshelfView(C.Structure):
    _fields_ = [
        ("design", Design),
        ("module_names", C.c_void_p),
        ("module_name_start", _i64),
        ("net_names", C.c_void_p),
        ("net_name_start", _i64),
        ("pin_direction", C.POINTER(C.c_int8)),
        ("row_orientation", _i32),
        ("declared_nodes", C.c_int64),
        ("declared_terminals", C.c_int64),
        ("declared_nets", C.c_int64),
        ("declared_pins", C.c_int64),
    ]


class Options(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("bins_x", C.c_int32),
        ("bins_y", C.c_int32),
        ("report_interval", C.c_int32),
        ("target_density", C.c_double),
        ("maximum_bin_overflow", C.c_double),
        ("initial_smoothing", C.c_double),
        ("final_smoothing", C.c_double),
        ("maximum_movement_in_bins", C.c_double),
        ("penalty_growth", C.c_double),
        ("optimizer", C.c_int32),
        ("maximum_backtracks", C.c_int32),
        ("backtracking_ratio", C.c_double),
        ("armijo_coefficient", C.c_double),
        ("maximum_momentum", C.c_double),
        ("initial_movement_in_bins", C.c_double),
        ("objective_increase_for_density", C.c_double),
        ("hpwl_growth_restart_threshold", C.c_double),
        ("density_stall_threshold", C.c_double),
        ("density_penalty_increase", C.c_double),
        ("density_penalty_decrease", C.c_double),
        ("minimum_density_penalty", C.c_double),
        ("maximum_density_penalty", C.c_double),
        ("smoothing_overflow_exponent", C.c_double),
        ("feasible_refinement_iterations", C.c_int32),
        ("pad0", C.c_int32),
        ("maximum_fillers", C.c_uint64),
        ("seed", C.c_uint64),
        ("rudy_columns", C.c_int32),
        ("rudy_rows", C.c_int32),
        ("rudy_minimum_span_in_bins", C.c_double),
        ("rudy_capacity_factor", C.c_double),
        ("rudy_softplus_temperature", C.c_double),
        ("rudy_penalty_model", C.c_int32),
        ("rudy_validation_bins", C.c_int32),
        ("rudy_validation_capacity_factor", C.c_double),
        ("routability_start_overflow", C.c_double),
        ("routability_weight_scale", C.c_double),
        ("routability_ramp_iterations", C.c_int32),
        ("density_field_boundary", C.c_int32),
        ("compute_backend", C.c_int32),
        ("cuda_device", C.c_int32),
        ("maximum_cuda_memory_bytes", C.c_uint64),
    ]


DENSITY_METRIC_FIELDS = [
    "total_overflow_area",
    "normalized_overflow",
    "maximum_density",
    "average_density",
    "total_charge_area",
    "normalization_area",
    "placeable_area",
    "dark_area",
]


class DensityMetrics(C.Structure):
    _fields_ = [(name, C.c_double) for name in DENSITY_METRIC_FIELDS]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name in DENSITY_METRIC_FIELDS}


class Evaluation(C.Structure):
    _fields_ = [
        ("hpwl", C.c_double),
        ("smooth_wirelength", C.c_double),
        ("electrostatic_energy", C.c_double),
        ("optimizer_density", DensityMetrics),
        ("design_density", DensityMetrics),
    ]


HISTORY_FIELDS = [
    "iteration", "hpwl", "overflow", "design_overflow", "smooth_wirelength", "density_energy", "objective",
    "penalty", "smoothing", "step_size", "maximum_displacement", "gradient_norm", "curvature", "rudy_energy",
    "rudy_proxy_overflow", "rudy_maximum_utilization", "rudy_weight", "backtracks", "momentum_restarted",
    "accepted", "best_checkpoint", "rudy_active",
]


class HistoryRow(C.Structure):
    _fields_ = [
        ("iteration", C.c_int32),
        ("backtracks", C.c_int32),
        ("hpwl", C.c_double),
        ("overflow", C.c_double),
        ("design_overflow", C.c_double),
        ("smooth_wirelength", C.c_double),
        ("density_energy", C.c_double),
        ("objective", C.c_double),
        ("penalty", C.c_double),
        ("smoothing", C.c_double),
        ("step_size", C.c_double),
        ("maximum_displacement", C.c_double),
        ("gradient_norm", C.c_double),
        ("curvature", C.c_double),
        ("rudy_energy", C.c_double),
        ("rudy_proxy_overflow", C.c_double),
        ("rudy_maximum_utilization", C.c_double),
        ("rudy_weight", C.c_double),
        ("momentum_restarted", C.c_int32),
        ("accepted", C.c_int32),
        ("best_checkpoint", C.c_int32),
        ("rudy_active", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name in HISTORY_FIELDS}


class Result(C.Structure):
    _fields_ = [
        ("hpwl_before", C.c_double),
        ("hpwl_after", C.c_double),
        ("overflow_before", C.c_double),
        ("overflow_after", C.c_double),
        ("completed_iterations", C.c_int32),
        ("accepted_iterations", C.c_int32),
        ("momentum_restarts", C.c_int32),
        ("rejected_candidates", C.c_int32),
        ("best_checkpoint_iteration", C.c_int32),
        ("restored_best_checkpoint", C.c_int32),
        ("best_checkpoint_hpwl", C.c_double),
        ("best_checkpoint_overflow", C.c_double),
        ("elapsed_seconds", C.c_double),
        ("compute_backend_used", C.c_int32),
        ("cuda_device_used", C.c_int32),
        ("cuda_reserved_memory_bytes", C.c_uint64),
        ("history_count", C.c_int32),
        ("evaluations", C.c_int32),
        ("rudy_energy_after", C.c_double),
        ("rudy_horizontal_capacity", C.c_double),
        ("rudy_vertical_capacity", C.c_double),
        ("rudy_proxy_overflow_after", C.c_double),
        ("rudy_maximum_utilization_after", C.c_double),
        ("rudy_p95_utilization_after", C.c_double),
        ("rudy_validation_energy_after", C.c_double),
        ("rudy_validation_proxy_overflow_after", C.c_double),
        ("rudy_validation_maximum_utilization_after", C.c_double),
        ("rudy_validation_p95_utilization_after", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Layout(C.Structure):
    _fields_ = [
        ("particle_count", C.c_int64),
        ("movable_count", C.c_int64),
        ("particle_width", _d),
        ("particle_height", _d),
        ("particle_layer", _i32),
        ("particle_pin_count", _i32),
        ("net_count", C.c_int32),
        ("pad0", C.c_int32),
        ("net_weight", _d),
        ("net_pin_start", _i64),
        ("pin_count", C.c_int64),
        ("pin_particle", _i32),
        ("pin_x", _d),
        ("pin_y", _d),
        ("bins_x", C.c_int32),
        ("bins_y", C.c_int32),
        ("region_llx", C.c_double),
        ("region_lly", C.c_double),
        ("region_urx", C.c_double),
        ("region_ury", C.c_double),
        ("target_density", C.c_double),
        ("static_fixed_area", _d),
        ("static_dark_area", _d),
    ]


class JobStats(C.Structure):
    _fields_ = [
        ("queued_seconds", C.c_double),
        ("run_seconds", C.c_double),
        ("latency_seconds", C.c_double),
        ("estimated_bytes", C.c_uint64),
        ("reserved_bytes", C.c_uint64),
        ("completed_iterations", C.c_int32),
        ("status", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64),
        ("completed", C.c_int64),
        ("failed", C.c_int64),
        ("iterations", C.c_int64),
        ("workers", C.c_int32),
        ("peak_running", C.c_int32),
        ("memory_budget", C.c_uint64),
        ("peak_reserved", C.c_uint64),
        ("seconds", C.c_double),
        ("batched", C.c_int32),
        ("batch_peak_round", C.c_int32),
        ("batch_rounds", C.c_int64),
        ("batch_evaluations", C.c_int64),
        ("batch_launches", C.c_int64),
        ("batch_busy_seconds", C.c_double),
        ("batch_device_seconds", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def _declare(lib: C.CDLL) -> C.CDLL:
    vp = C.c_void_p
    sig = {
        "mpgp_compiled": (C.c_int, []),
        "mpgp_abi_version": (C.c_int, []),
        "mpgp_last_error": (C.c_char_p, []),
        "mpgp_options_default": (None, [C.POINTER(Options)]),
        "mpgp_backend_create": (C.c_int, [C.POINTER(Layout), C.c_int, C.c_uint64, C.POINTER(vp), C.c_char_p,
                                          C.c_size_t]),
        "mpgp_backend_evaluate": (C.c_int, [vp, _d, C.c_double, C.c_int, C.POINTER(Evaluation), _d, _d]),
        "mpgp_backend_set_stall_probe": (C.c_int, [vp, C.c_int64]),
        "mpgp_backend_device": (C.c_int, [vp]),
        "mpgp_backend_reserved_bytes": (C.c_uint64, [vp]),
        "mpgp_backend_destroy": (None, [vp]),
        "mpgp_backend_density_layers": (C.c_int, [vp, _i64, _i64, _i64]),
        "mpgp_backend_field_solve": (C.c_int, [vp, _d, _d, _d, _d]),
        "mpgp_backend_rudy": (C.c_int, [vp, C.POINTER(Options), _d, C.c_double, C.c_double, C.c_int, _d, _d, _d]),
        "mpgp_random_placement": (C.c_int, [C.POINTER(Design), C.c_uint64, _d, _d]),
        "mpgp_detailed_options_default": (None, [C.POINTER(DetailedOptions)]),
        "mpgp_detailed_place": (C.c_int, [C.POINTER(Design), _i32, C.POINTER(DetailedOptions), _d, _d, _i32,
                                          C.POINTER(DetailedResult), C.c_char_p, C.c_size_t]),
        "mpgp_bookshelf_read": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(vp)]),
        "mpgp_bookshelf_get": (C.c_int, [vp, C.POINTER(BookshelfView)]),
        "mpgp_bookshelf_destroy": (None, [vp]),
        "mpgp_wirelength_noalloc": (C.c_int, [vp, vp, vp, vp, vp, C.c_int32, C.c_int32, vp, vp, C.c_int32,
                                              C.c_double, vp, vp, vp]),
        "mpgp_global_place": (C.c_int, [C.POINTER(Design), C.POINTER(Options), _d, _d, C.POINTER(Result),
                                        C.POINTER(HistoryRow), C.c_int32]),
        "mpgp_session_create": (C.c_int, [C.POINTER(Design), C.POINTER(Options), C.POINTER(vp)]),
        "mpgp_session_step": (C.c_int, [vp, C.c_int32, _i32, _i32]),
        "mpgp_session_finish": (C.c_int, [vp, _d, _d, C.POINTER(Result), C.POINTER(HistoryRow), C.c_int32]),
        "mpgp_setup_create": (C.c_int, [C.POINTER(Design), C.POINTER(Options), C.POINTER(vp)]),
        "mpgp_setup_particles": (C.c_int, [vp, _i64, _i64, _d, _d, _d, _d, _i32, _d]),
        "mpgp_setup_static_density": (C.c_int, [vp, _d, _d]),
        "mpgp_setup_destroy": (None, [vp]),
        "mpgp_session_positions": (C.c_int, [vp, _d]),
        "mpgp_session_kernel_launches": (C.c_int64, [vp]),
        "mpgp_kernel_kind_count": (C.c_int, []),
        "mpgp_kernel_kind_name": (C.c_char_p, [C.c_int]),
        "mpgp_session_set_profiling": (C.c_int, [vp, C.c_uint32]),
        "mpgp_session_kernel_stats": (C.c_int, [vp, _i64, _d, C.c_int32]),
        "mpgp_session_reset_kernel_stats": (C.c_int, [vp]),
        "mpgp_session_transfer_bytes": (C.c_int, [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "mpgp_session_stream": (vp, [vp]),
        "mpgp_session_destroy": (None, [vp]),
        "mpgp_estimate_bytes": (C.c_int, [C.POINTER(Design), C.POINTER(Options), C.POINTER(C.c_uint64)]),
        "mpgp_tuning_set_splits": (C.c_int, [_i32, _i32, C.c_int32]),
        "mpgp_tuning_get_splits": (C.c_int, [_i32, _i32, C.c_int32, _i32]),
        "mpgp_server_create": (C.c_int, [C.c_int, C.c_uint64, C.c_int32, C.POINTER(vp)]),
        "mpgp_server_create_mode": (C.c_int, [C.c_int, C.c_uint64, C.c_int32, C.c_int32, C.POINTER(vp)]),
        "mpgp_server_submit": (C.c_int, [vp, C.POINTER(Design), C.POINTER(Options), C.POINTER(C.c_int64)]),
        "mpgp_server_wait": (C.c_int, [vp, C.c_int64, C.c_double, _i32]),
        "mpgp_server_take": (C.c_int, [vp, C.c_int64, _d, _d, C.POINTER(Result), C.POINTER(HistoryRow), C.c_int32,
                                       C.POINTER(JobStats)]),
        "mpgp_server_stats_get": (C.c_int, [vp, C.POINTER(ServerStats)]),
        "mpgp_server_destroy": (None, [vp]),
        "mpgp_batch_place": (C.c_int, [C.c_int32, C.POINTER(Design), C.POINTER(Options), C.c_int, C.c_int32,
                                       C.c_int32, C.c_uint64, C.POINTER(_d), C.POINTER(_d), C.POINTER(Result),
                                       C.POINTER(JobStats), C.POINTER(ServerStats)]),
    }
    for name, (restype, argtypes) in sig.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    return lib


_LIB: C.CDLL | None = None


def load_library() -> C.CDLL:
    """Loads libmpgp.so from the package directory; raises if it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIBRARY_PATH.is_file():
        raise RuntimeError(
            f"libmpgp.so is not built ({LIBRARY_PATH}); run `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `python -m myplacement_b200.build`. The engine has no CPU fallback.")
    _LIB = _declare(C.CDLL(str(LIBRARY_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL))
    return _LIB


class EngineError(RuntimeError):
    """A non-zero status from the engine, with its last-error message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"mpgp status {status}: {message}")
        self.status = status


class ParseError(EngineError):
    """Malformed BookShelf input: the reference's myplacement::ParseError."""


def check(status: int) -> None:
    if status != MPGP_OK:
        message = load_library().mpgp_last_error().decode(errors="replace")
        raise (ParseError if status == MPGP_ERR_PARSE else EngineError)(status, message)
