"""Detailed placement by window reordering on the device.

``DetailedPlacer().run(design, options)`` is the reference's
``DetailedPlacer::run`` (include/myplacement/placement/DetailedPlacer.hpp:59-63)
with the CUDA backend (src/placement/cuda/CudaDetailedPlacementBackend.cu):
every order of four consecutive cells of a row segment is evaluated on the
B200 and accepted by the reference's rule, on a legal placement.  It returns
the placed design and the DetailedPlacementResult fields; where the device
backend declines (options other than a four-cell window reorder, no device) it
raises :class:`EngineError` with status MPGP_ERR_UNAVAILABLE and the reason,
as the reference raises std::invalid_argument for ``--detailed-backend cuda``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import check, load_library
from .design import Design

__all__ = ["DetailedPlacer", "default_detailed_options"]


def default_detailed_options(**overrides) -> _abi.DetailedOptions:
    """DetailedPlacementOptions defaults with the window reorder selected, device 0."""
    options = _abi.DetailedOptions()
    load_library().mpgp_detailed_options_default(C.byref(options))
    for key, value in overrides.items():
        setattr(options, key, value)
    return options


class DetailedPlacer:
    def run(self, design: Design, options: _abi.DetailedOptions | None = None,
            row_orientation: np.ndarray | None = None) -> tuple[Design, dict]:
        options = options if options is not None else default_detailed_options()
        if row_orientation is None and design.bookshelf is not None:
            row_orientation = getattr(design.bookshelf, "row_orientation", None)
        rows = None if row_orientation is None else np.ascontiguousarray(row_orientation, dtype=np.int32)
        x = np.empty(design.module_count)
        y = np.empty(design.module_count)
        orientation = np.empty(design.module_count, np.int32)
        result = _abi.DetailedResult()
        reason = C.create_string_buffer(1024)
        s = design.as_c()
        check(load_library().mpgp_detailed_place(
            C.byref(s), None if rows is None else rows.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(options),
            x.ctypes.data_as(C.POINTER(C.c_double)), y.ctypes.data_as(C.POINTER(C.c_double)),
            orientation.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(result), reason, len(reason)))
        placed = design.copy_with_positions(x, y)
        placed.module_orientation = orientation
        return placed, result.as_dict()
