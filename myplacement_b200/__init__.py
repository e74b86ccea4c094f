"""B200-native global placement for MyPlacement's adaptive + neumann + course_eplace_v1 method.

The engine is the native library ``libmpgp.so`` (C ABI in include/mpgp.h,
hand-written sm_100a CUDA kernels); this package is its host-side mirror of the
reference's GlobalPlacer / CudaPlacementBackend interface plus the seeded
synthetic designs the engine is measured on.
"""
from ._abi import EngineError, ParseError, load_library
from .bookshelf import BookshelfParser, read_bookshelf, write_bookshelf
from .design import Design, synthetic_design, workload
from .detailed import DetailedPlacer, default_detailed_options
from .placer import (BackendLayout, CudaPlacementBackend, GlobalPlacer, PlacementResult, PlacementServer, Session,
                     batch_place, build_layout, default_options, estimate_bytes, host_setup, random_placement,
                     try_create_backend)

__all__ = [
    "BackendLayout", "BookshelfParser", "CudaPlacementBackend", "Design", "DetailedPlacer", "EngineError",
    "GlobalPlacer", "default_detailed_options",
    "ParseError", "PlacementResult", "PlacementServer", "Session", "batch_place", "build_layout", "estimate_bytes",
    "default_options", "host_setup", "load_library", "random_placement", "read_bookshelf", "synthetic_design",
    "try_create_backend", "workload", "write_bookshelf",
]
